"""GPU parity tests of the tensor-core forms (split-BF16 or single-BF16 tcgen05
contraction + FP64 recheck of the rows inside the form's error band): responses
must equal the FP64 oracle's exactly."""
import ctypes

import numpy as np
import pytest
import torch

from helpers import centroid_rel_err, rel_close
from onedal_b200 import _native, kmeans, workloads
from oracle import restated

pytestmark = pytest.mark.gpu


# the split form (three BF16 products per k-step) and the single-product form: both
# recheck every row inside their own error band in FP64
FORMS = [kmeans.compute_form.bf16x3, kmeans.compute_form.bf16]


def tc_desc(k, T=100, eps=0.0, form=kmeans.compute_form.bf16x3):
    return (kmeans.descriptor(np.float32).set_cluster_count(k).set_max_iteration_count(T)
            .set_accuracy_threshold(eps).set_compute_form(form))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n,d,k", [(1, 1, 1), (129, 3, 5), (1000, 7, 130), (4099, 37, 257), (3000, 130, 64),
                                   (2048, 256, 300), (5000, 64, 1024), (777, 128, 129)])
def test_infer_exact_vs_fp64_oracle(n, d, k, form):
    rng = np.random.default_rng(n * 7 + d + k)
    X = (rng.standard_normal((n, d)) * 3).astype(np.float32)
    C = (rng.standard_normal((k, d)) * 3).astype(np.float32)
    if k <= n:
        C = X[rng.choice(n, k, replace=False)] + (0.05 * rng.standard_normal((k, d))).astype(np.float32)
    dsc = tc_desc(k, form=form).set_result_options(kmeans.result_options.compute_exact_objective_function)
    r = kmeans.infer(dsc, kmeans.model(C), X)
    lab64, _, _ = restated.assign_f32_in_f64(X, C)
    assert (r.get_responses().ravel() == lab64).all()
    obj64 = restated.objective(X.astype(np.float64), C.astype(np.float64), lab64)
    assert rel_close(r.get_objective_function_value(), obj64, 1e-6)


@pytest.mark.parametrize("form", FORMS)
def test_near_ties_are_rechecked(form):
    """Rows placed exactly between two centroids (+ tiny noise) must all follow the
    FP64 oracle, including exact ties (lowest index)."""
    rng = np.random.default_rng(1)
    k, d = 64, 128
    C = rng.uniform(-5, 5, (k, d)).astype(np.float32)
    a = rng.integers(0, k, 4000)
    b = (a + rng.integers(1, k, 4000)) % k
    mid = 0.5 * (C[a].astype(np.float64) + C[b].astype(np.float64))
    X = (mid + 1e-4 * rng.standard_normal(mid.shape)).astype(np.float32)
    X[:64] = C[:64]  # rows equal to a centroid
    r = kmeans.infer(tc_desc(k, form=form), kmeans.model(C), X)
    lab64, _, _ = restated.assign_f32_in_f64(X, C)
    assert (r.get_responses().ravel() == lab64).all()
    assert r.stats.rechecked_rows > 1000


@pytest.mark.parametrize("form", FORMS)
def test_duplicate_centroids_tie_to_lowest_index(form):
    rng = np.random.default_rng(2)
    C = rng.standard_normal((10, 32)).astype(np.float32)
    C[7] = C[3]
    X = np.repeat(C[3:4], 50, axis=0) + (1e-3 * rng.standard_normal((50, 32))).astype(np.float32)
    r = kmeans.infer(tc_desc(10, form=form), kmeans.model(C), X)
    lab64, _, _ = restated.assign_f32_in_f64(X, C)
    assert (r.get_responses().ravel() == lab64).all()
    assert not (r.get_responses().ravel() == 7).any()


@pytest.mark.parametrize("form", FORMS)
def test_lockstep_precision_shape(form):
    """Reduced precision-shaped workload (d=128, k=512, 10% bisector near-ties), three
    iterations in lock-step with the FP64 oracle from the same C^(t)."""
    X, C0 = workloads.make(workloads.Workload("precision", 40000, 128, 512, 3, 0.0, 21), "cpu", 40000)
    X = X.numpy()
    ctx = _native.context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    Xd = torch.from_numpy(X).cuda()
    Cd = C0.cuda()
    out = torch.empty_like(Cd)
    lab = torch.empty(X.shape[0], dtype=torch.int32, device="cuda")
    shift, ne = ctypes.c_double(), ctypes.c_int64()
    for t in range(3):
        C_in = Cd.cpu().numpy()
        ctx.check(ctx.lib.kmb_lloyd_step(ctx.handle, _native.KMB_F32, Xd.data_ptr(), X.shape[0], 128, Cd.data_ptr(),
                                         512, form, 1, out.data_ptr(), lab.data_ptr(),
                                         ctypes.byref(shift), ctypes.byref(ne)))
        torch.cuda.synchronize()
        C64, lab64, shift64, ne64, _ = restated.step(X.astype(np.float64), C_in.astype(np.float64))
        assert (lab.cpu().numpy() == lab64).all(), f"iteration {t}"
        if ne64 == 0:
            assert centroid_rel_err(C64, out.cpu().numpy()) < 1e-5
        Cd.copy_(out)


@pytest.mark.parametrize("form", FORMS)
def test_train_equals_plain_form_with_recheck(form):
    """Both forms give FP64-oracle responses every iteration and share the
    deterministic update, so whole trainings agree bit for bit."""
    X, C0 = workloads.make(workloads.Workload("precision", 60000, 64, 200, 8, 0.0, 22), "cpu", 60000)
    X, C0 = X.numpy(), C0.numpy()
    a = kmeans.train(tc_desc(200, 8, form=form), X, C0)
    p = kmeans.descriptor(np.float32).set_cluster_count(200).set_max_iteration_count(8).set_recheck(True)
    b = kmeans.train(p, X, C0)
    assert a.get_iteration_count() == b.get_iteration_count()
    np.testing.assert_array_equal(a.get_responses(), b.get_responses())
    np.testing.assert_array_equal(a.get_model().get_centroids(), b.get_model().get_centroids())
    assert a.get_objective_function_value() == b.get_objective_function_value()


@pytest.mark.parametrize("form", FORMS)
def test_gold_data_tensor_core_form(form):
    from helpers import find_match_centroids, load_json
    g = load_json("gold.json")
    X = np.array(g["data"], np.float32).reshape(100, 3)
    C0 = np.array(g["initial_centroids"], np.float32).reshape(3, 3)
    r = kmeans.train(tc_desc(3, 100, 0.0, form=form), X, C0)
    exp = np.array(g["expected_centroids"]).reshape(3, 3)
    m = find_match_centroids(exp, r.get_model().get_centroids())
    assert centroid_rel_err(exp, r.get_model().get_centroids(), m) < 1e-6
    assert rel_close(r.get_objective_function_value(), g["expected_objective"], 1e-6)
    assert (m[r.get_responses().ravel()] == np.array(g["expected_responses"])).all()


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n,d,k,T", [(40000, 128, 512, 6), (30000, 96, 300, 10)])
def test_train_multi_iteration_equals_plain_form(n, d, k, T, form):
    """From the second iteration on, the tensor-core epilogue skips clusters below a
    lower bound built from the previous labels, distances and centroid shifts; whole
    trainings must still equal the plain form with recheck bit for bit."""
    X, C0 = workloads.make(workloads.Workload("precision", n, d, k, T, 0.0, 23 + d), "cpu", n)
    X, C0 = X.numpy(), C0.numpy()
    a = kmeans.train(tc_desc(k, T, form=form), X, C0)
    p = kmeans.descriptor(np.float32).set_cluster_count(k).set_max_iteration_count(T).set_recheck(True)
    b = kmeans.train(p, X, C0)
    assert a.get_iteration_count() == b.get_iteration_count()
    np.testing.assert_array_equal(a.get_responses(), b.get_responses())
    np.testing.assert_array_equal(a.get_model().get_centroids(), b.get_model().get_centroids())
    assert a.get_objective_function_value() == b.get_objective_function_value()


@pytest.mark.parametrize("form", FORMS)
def test_train_with_reseeds_equals_plain_form(form):
    """Duplicate initial centroids empty clusters in the first iterations; reseeded
    clusters move far, which the prior bound must absorb."""
    rng = np.random.default_rng(24)
    centres = rng.uniform(-5, 5, (64, 48))
    X = (centres[rng.integers(0, 64, 20000)] + rng.standard_normal((20000, 48))).astype(np.float32)
    C0 = np.repeat(X[:16], 4, axis=0).copy()
    a = kmeans.train(tc_desc(64, 12, form=form), X, C0)
    p = kmeans.descriptor(np.float32).set_cluster_count(64).set_max_iteration_count(12).set_recheck(True)
    b = kmeans.train(p, X, C0)
    assert a.get_iteration_count() == b.get_iteration_count()
    np.testing.assert_array_equal(a.get_responses(), b.get_responses())
    np.testing.assert_array_equal(a.get_model().get_centroids(), b.get_model().get_centroids())


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n,d,k", [(1, 5, 3), (200, 64, 129), (385, 128, 300), (20000, 128, 1024), (9000, 200, 520)])
def test_cta_pair_and_single_cta_kernels_agree(n, d, k, monkeypatch, form):
    """The assignment runs on single CTAs by default and on CTA pairs
    (cta_group::2, 256-row units, each CTA loading half of every centroid panel)
    with KMB_TC_PAIR=1; both must give the FP64 oracle's responses and the same objective,
    for row counts that leave the last pair half empty and both cluster-tile widths."""
    rng = np.random.default_rng(n + d + k)
    X = (rng.standard_normal((n, d)) * 2).astype(np.float32)
    C = (rng.standard_normal((k, d)) * 2).astype(np.float32)
    dsc = tc_desc(k, form=form).set_result_options(kmeans.result_options.compute_exact_objective_function)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("KMB_TC_PAIR", mode)
        r = kmeans.infer(dsc, kmeans.model(C), X)
        out[mode] = (r.get_responses().ravel().copy(), r.get_objective_function_value())
    lab64, _, _ = restated.assign_f32_in_f64(X, C)
    assert (out["1"][0] == lab64).all()
    assert (out["0"][0] == lab64).all()
    assert rel_close(out["1"][1], out["0"][1], 1e-12)


@pytest.mark.parametrize("form", FORMS)
def test_cta_pair_training_matches_single_cta_training(monkeypatch, form):
    """A few Lloyd iterations (prior-bound filter active from the second one) give
    bit-identical centroids and responses on CTA pairs and on single CTAs."""
    X, C0 = workloads.make(workloads.Workload("precision", 50000, 128, 512, 4, 0.0, 21), "cpu", 50000)
    X, C0 = X.numpy(), C0.numpy()
    res = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("KMB_TC_PAIR", mode)
        r = kmeans.train(tc_desc(512, 4, form=form), X, C0)
        res[mode] = (r.get_model().get_centroids().copy(), r.get_responses().ravel().copy())
    np.testing.assert_array_equal(res["1"][0], res["0"][0])
    np.testing.assert_array_equal(res["1"][1], res["0"][1])
