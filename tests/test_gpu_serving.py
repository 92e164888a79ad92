"""GPU tests of the serving loop: every result is the same alone and in the mix
(responses and trained centroids exactly equal to the single-call API), the HBM
budget is respected, and concurrent requests are batched into shared launches."""
import threading

import numpy as np
import pytest

from onedal_b200 import _native, kmeans
from onedal_b200.serving import KMeansServer

pytestmark = pytest.mark.gpu


def _models(rng, count=6):
    out = []
    for _ in range(count):
        k = int(rng.choice([16, 40, 128, 300, 700]))
        d = int(rng.choice([32, 64, 128, 256]))
        out.append(rng.uniform(-1, 1, (k, d)).astype(np.float32))
    return out


def _alone_infer(C, X, form=_native.KMB_FORM_PLAIN):
    """The same infer alone, through kmeans.infer in the given form (explicit: the mirror's
    default form is auto)."""
    d = kmeans.descriptor(np.float32).set_cluster_count(C.shape[0])
    d = d.set_compute_form(kmeans.compute_form.bf16x3 if form == _native.KMB_FORM_BF16X3
                           else kmeans.compute_form.plain)
    return kmeans.infer(d, kmeans.model(C), X).get_responses().ravel()


def test_mixed_requests_equal_alone():
    rng = np.random.default_rng(31)
    models = _models(rng)
    with KMeansServer(hbm_budget_bytes=8 << 30, lanes=3, trainers=2) as srv:
        ids = [srv.add_model(C) for C in models]
        reqs = []
        for i in range(120):
            m = int(rng.integers(0, len(models)))
            n = int(min(200_000, max(1, rng.lognormal(np.log(2048), 1.5))))
            X = rng.standard_normal((n, models[m].shape[1])).astype(np.float32)
            reqs.append(("infer", m, X, srv.submit_infer(ids[m], X), srv.infer_form(ids[m], n)))
            if i % 10 == 0:
                k = int(rng.integers(4, 64))
                nt = int(rng.integers(max(k, 1000), 20_000))
                centres = rng.uniform(-10, 10, (k, 16))
                Xt = (centres[rng.integers(0, k, nt)] + rng.standard_normal((nt, 16))).astype(np.float32)
                reqs.append(("train", k, Xt, srv.submit_train(Xt, Xt[:k], 15), None))
        for kind, m, X, r, form in reqs:
            out, lat = srv.wait(r, timeout=120)
            assert lat > 0
            if kind == "infer":
                np.testing.assert_array_equal(out, _alone_infer(models[m], X, form))
            else:
                C, lab = out
                d = kmeans.descriptor(np.float32).set_cluster_count(m).set_max_iteration_count(15)
                alone = kmeans.train(d, X, X[:m])
                np.testing.assert_array_equal(C, alone.get_model().get_centroids())
                np.testing.assert_array_equal(lab, alone.get_responses().ravel())
        st = srv.stats()
        assert st["failed"] == 0
        assert st["completed"] == len(reqs)
        assert st["batches"] >= 1
        n_tc = sum(1 for q in reqs if q[4] == _native.KMB_FORM_BF16X3)
        assert st["tensor_core_requests"] == n_tc


def test_large_requests_use_tensor_cores_and_match_fp64_oracle():
    """Large infer requests go to the tensor-core worker; their responses are the FP64
    oracle's and equal the single-call BF16x3 infer, also while small requests run."""
    from oracle import restated
    rng = np.random.default_rng(34)
    C = rng.uniform(-1, 1, (128, 32)).astype(np.float32)
    small_C = rng.uniform(-1, 1, (40, 32)).astype(np.float32)
    with KMeansServer(hbm_budget_bytes=8 << 30, lanes=2, trainers=1) as srv:
        big, small = srv.add_model(C), srv.add_model(small_C)
        n_big = 1_100_000  # 1.1e6 * 128 * 64 >= 2^33 multiply-adds; five row chunks of 2^18
        assert srv.infer_form(big, n_big) == _native.KMB_FORM_BF16X3
        assert srv.infer_form(big, 1000) == _native.KMB_FORM_PLAIN
        Xb = rng.standard_normal((n_big, 32)).astype(np.float32)
        rb = srv.submit_infer(big, Xb)
        smalls = [(rng.standard_normal((int(rng.integers(1, 3000)), 32)).astype(np.float32)) for _ in range(30)]
        rs = [srv.submit_infer(small, X) for X in smalls]
        lab, _ = srv.wait(rb, timeout=120)
        lab64, _, _ = restated.assign_f32_in_f64(Xb, C)
        np.testing.assert_array_equal(lab, lab64)
        np.testing.assert_array_equal(lab, _alone_infer(C, Xb, _native.KMB_FORM_BF16X3))
        for X, r in zip(smalls, rs):
            out, _ = srv.wait(r, timeout=60)
            np.testing.assert_array_equal(out, _alone_infer(small_C, X))
        assert srv.stats()["tensor_core_requests"] == 1


def test_requests_arriving_during_a_batch_share_a_launch():
    """Continuous batching: with one lane busy on a long request, requests that arrive
    meanwhile are admitted together into the next grouped launch."""
    rng = np.random.default_rng(35)
    C = rng.uniform(-1, 1, (1024, 64)).astype(np.float32)
    with KMeansServer(hbm_budget_bytes=8 << 30, lanes=1, trainers=1) as srv:
        mid = srv.add_model(C)
        long_rows = rng.standard_normal((120_000, 64)).astype(np.float32)
        assert srv.infer_form(mid, long_rows.shape[0]) == _native.KMB_FORM_PLAIN
        first = srv.submit_infer(mid, long_rows)
        smalls = [rng.standard_normal((int(rng.integers(1, 500)), 64)).astype(np.float32) for _ in range(40)]
        reqs = [srv.submit_infer(mid, X) for X in smalls]
        lab, _ = srv.wait(first, timeout=60)
        np.testing.assert_array_equal(lab, _alone_infer(C, long_rows))
        for X, r in zip(smalls, reqs):
            out, _ = srv.wait(r, timeout=60)
            np.testing.assert_array_equal(out, _alone_infer(C, X))
        st = srv.stats()
        assert st["batched_requests"] == 41
        assert st["batches"] < st["batched_requests"]


def test_budget_is_respected_and_queued_requests_complete():
    rng = np.random.default_rng(32)
    C = rng.uniform(-1, 1, (64, 64)).astype(np.float32)
    budget = 48 << 20
    with KMeansServer(hbm_budget_bytes=budget, lanes=2, trainers=1) as srv:
        mid = srv.add_model(C)
        X = rng.standard_normal((60_000, 64)).astype(np.float32)  # ~16 MB of device bytes each
        reqs = [srv.submit_infer(mid, X) for _ in range(12)]
        ref = _alone_infer(C, X)
        for r in reqs:
            lab, _ = srv.wait(r, timeout=120)
            np.testing.assert_array_equal(lab, ref)
        st = srv.stats()
        assert st["peak_in_use_bytes"] <= budget
        assert st["in_use_bytes"] == 0


def test_submit_from_many_threads():
    rng = np.random.default_rng(33)
    C = rng.uniform(-1, 1, (200, 32)).astype(np.float32)
    with KMeansServer(hbm_budget_bytes=4 << 30) as srv:
        mid = srv.add_model(C)
        errors = []

        def worker(seed):
            g = np.random.default_rng(seed)
            try:
                for _ in range(20):
                    X = g.standard_normal((int(g.integers(1, 5000)), 32)).astype(np.float32)
                    lab, _ = srv.wait(srv.submit_infer(mid, X), timeout=60)
                    np.testing.assert_array_equal(lab, _alone_infer(C, X))
            except Exception as e:  # pragma: no cover - reported below
                errors.append(e)

        ts = [threading.Thread(target=worker, args=(s,)) for s in range(6)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        assert not errors, errors[0]
