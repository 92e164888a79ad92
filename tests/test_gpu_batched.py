"""GPU tests of the batched form: many uneven problems trained by one persistent
grouped kernel must reproduce each problem trained alone (kmb_lloyd_iterate,
plain form) bit for bit -- centroids, responses and iteration counts -- and the
FP64 oracle's responses under the returned centroids."""
import ctypes

import numpy as np
import pytest
import torch

from onedal_b200 import _native
from onedal_b200.batched import batched_train
from oracle import restated

pytestmark = pytest.mark.gpu


def _problems(count, seed):
    g = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(np.exp(g.uniform(np.log(1000), np.log(40_000))))
        d = int(g.choice([5, 8, 13, 16, 32, 64, 100]))
        k = int(np.exp(g.uniform(np.log(4), np.log(200))))
        c = g.uniform(-10, 10, (k, d))
        X = (c[g.integers(0, k, n)] + g.standard_normal((n, d))).astype(np.float32)
        out.append((X, X[g.choice(n, k, replace=False)].copy()))
    return out


def _alone(X, C0, T):
    ctx = _native.context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    Xd = torch.from_numpy(X).cuda()
    C = torch.from_numpy(C0).cuda()
    lab = torch.empty(X.shape[0], dtype=torch.int32, device="cuda")
    p = _native.kmb_params(C0.shape[0], T, 0.0, _native.KMB_FORM_PLAIN, 0)
    it = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_lloyd_iterate(ctx.handle, _native.KMB_F32, Xd.data_ptr(), X.shape[0], X.shape[1],
                                        C.data_ptr(), ctypes.byref(p), lab.data_ptr(), ctypes.byref(it), None))
    torch.cuda.synchronize()
    return C.cpu().numpy(), lab.cpu().numpy(), it.value


@pytest.mark.parametrize("use_graph", [True, False])
def test_batched_matches_alone(use_graph):
    probs = _problems(40, 51)
    T = 12
    res, info = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()) for X, C0 in probs], T,
                              use_graph=use_graph)
    assert info["problems"] == 40 and info["variants"] >= 1
    for (X, C0), (C, lab, it) in zip(probs, res):
        Ca, laba, ita = _alone(X, C0, T)
        assert it == ita
        np.testing.assert_array_equal(lab.cpu().numpy(), laba)
        np.testing.assert_array_equal(C.cpu().numpy(), Ca)


def test_batched_many_problems_match_alone():
    """600 small problems (more work items than the grid has CTAs in every phase);
    a seeded fifth of them checked against the alone path."""
    probs = _problems(600, 54)
    probs = [(X[: max(C0.shape[0] * 4, X.shape[0] // 8)], C0) for X, C0 in probs]
    res, info = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()) for X, C0 in probs], 25)
    assert info["problems"] == 600
    assert info["total_iterations"] == sum(it for _, _, it in res)
    for i in np.random.default_rng(55).choice(600, 120, replace=False):
        X, C0 = probs[i]
        C, lab, it = res[i]
        Ca, laba, ita = _alone(X, C0, 25)
        assert it == ita, i
        np.testing.assert_array_equal(lab.cpu().numpy(), laba)
        np.testing.assert_array_equal(C.cpu().numpy(), Ca)


def test_batched_converged_problems_stop_and_match_oracle():
    """eps = 0: each problem stops at its fixed point, at the same iteration as
    alone. Every returned model is a fixed point of the FP64 oracle's update (one
    oracle step from it reproduces it) up to FP32 near-tie labels; most problems
    reach the oracle's own fixed point."""
    probs = _problems(12, 52)
    res, _ = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()) for X, C0 in probs], 100)
    same = 0
    for (X, C0), (C, lab, it) in zip(probs, res):
        assert it < 100  # converged
        Ca, laba, ita = _alone(X, C0, 100)
        assert it == ita
        C = C.cpu().numpy()
        lab = lab.cpu().numpy()
        np.testing.assert_array_equal(C, Ca)
        C1, lab64, _, ne, _ = restated.step(X.astype(np.float64), C.astype(np.float64))
        assert (lab64 != lab).mean() < 1e-3
        if (lab64 == lab).all() and ne == 0:
            np.testing.assert_allclose(C1, C, rtol=1e-5, atol=1e-5)
        ref_C, _, _, ref_it = restated.train(X.astype(np.float64), C0.astype(np.float64), 100, 0.0)
        if it == ref_it and np.allclose(C, ref_C, rtol=1e-5, atol=1e-5):
            same += 1
    assert same >= 6


def test_batched_empty_cluster_reseed():
    """Six clusters seeded on one row: five empty in the first update, reseeded with
    the farthest rows in (distance descending, row ascending) order, as alone."""
    g = np.random.default_rng(53)
    X = (g.standard_normal((3000, 8)) * g.uniform(0.5, 3, 8)).astype(np.float32)
    C0 = (np.repeat(X[:1], 6, axis=0) + 1e-3 * np.arange(6)[:, None]).astype(np.float32)
    X2 = np.repeat(X[:400], 2, axis=0)  # duplicated rows: equal distances, ties broken by row
    C2 = np.repeat(X2[:1], 9, axis=0).astype(np.float32)
    res, _ = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()),
                            (torch.from_numpy(X2).cuda(), torch.from_numpy(C2).cuda())], 3)
    for (Xi, Ci), (C, lab, it) in zip([(X, C0), (X2, C2)], res):
        Ca, laba, ita = _alone(Xi, Ci, 3)
        assert it == ita
        np.testing.assert_array_equal(C.cpu().numpy(), Ca)
        np.testing.assert_array_equal(lab.cpu().numpy(), laba)


def test_batched_rejects_out_of_range_problems():
    X = torch.zeros((100, 4), device="cuda")
    with pytest.raises(Exception):
        batched_train([(X, torch.zeros((300, 4), device="cuda"))], 3)  # k > 256
    with pytest.raises(Exception):
        batched_train([(X[:10], torch.zeros((20, 4), device="cuda"))], 3)  # k > n
