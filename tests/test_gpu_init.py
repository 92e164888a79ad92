"""GPU tests of the k-means++ default initialisation (kmb_init_plusplus through the C ABI).

The reference picks centers by sampling rows of the data, so the bar is exact: the
chosen centers are bit-identical rows of X, the same rows the reference build picked
(tests/golden/daal_ref_plusplus.npz) and the same rows the oracle picks
(oracle/kmeans_init_oracle.cpp) for any seed.
"""
import os
import sys

import numpy as np
import pytest
import torch

from helpers import GOLDEN, centroid_rel_err, rel_close
from onedal_b200 import kmeans
from oracle import restated

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.float32]


def _fixture_inputs():
    sys.path.insert(0, GOLDEN)
    from make_golden import plusplus_cases
    z = np.load(os.path.join(GOLDEN, "example_dense.npz"))
    return plusplus_cases() + [("example", z["X"], 20)]


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_plusplus_matches_reference_fixtures(tag, dt):
    z = np.load(os.path.join(GOLDEN, "daal_ref_plusplus.npz"))
    for name, X, k in _fixture_inputs():
        X = X.astype(dt)
        C = kmeans.init_plusplus(X, k, dt)
        assert C.dtype == dt
        assert np.array_equal(C, z[f"C_{name}_{tag}"]), name


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("n,d,k,seed", [(1, 1, 1, 1), (511, 3, 511, 2), (513, 17, 40, 3), (5000, 130, 257, 4),
                                         (70001, 9, 64, 5), (300000, 32, 16, 6), (300007, 40, 8, 7),
                                         (2500001, 4, 12, 8)])
def test_plusplus_matches_oracle(dt, n, d, k, seed):
    """Ragged block counts (n around the 512-row block), k == n, rows narrower and wider
    than one 128-byte segment of the distance kernel, and 2.5M rows (more block sums than
    one shared-memory chunk of the selection kernel holds)."""
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((n, d)) * rng.uniform(0.1, 4.0, d)).astype(dt)
    for s in (777777, seed):
        C = kmeans.init_plusplus(X, k, dt, seed=s)
        Co, rows = restated.init_plusplus(X, k, s)
        assert np.array_equal(C, Co), (n, d, k, s)


@pytest.mark.parametrize("dt", DTYPES)
def test_plusplus_duplicates_and_pool_refill(dt, monkeypatch):
    """Integer grids with exactly k distinct rows force resampling; a one-entry resample
    pool makes every resample go through the host refill and round resume."""
    rng = np.random.default_rng(11)
    X = rng.integers(0, 4, (6000, 2)).astype(dt)
    ref = restated.init_plusplus(X, 16, 777777)[0]
    assert np.array_equal(kmeans.init_plusplus(X, 16, dt), ref)
    monkeypatch.setenv("KMB_PLUSPLUS_POOL", "1")
    assert np.array_equal(kmeans.init_plusplus(X, 16, dt), ref)
    Y = np.round(3 * rng.standard_normal((20000, 3))).astype(dt)
    for s in (1, 2, 3):
        assert np.array_equal(kmeans.init_plusplus(Y, 200, dt, seed=s), restated.init_plusplus(Y, 200, s)[0])


@pytest.mark.parametrize("dt", DTYPES)
def test_plusplus_fewer_distinct_rows_than_k(dt):
    """The reference's resampling never ends here; this path reports invalid_argument."""
    X = np.repeat(np.arange(3, dtype=dt)[:, None], 100, axis=0)
    assert np.array_equal(kmeans.init_plusplus(X, 3, dt), restated.init_plusplus(X, 3)[0])
    with pytest.raises(kmeans.invalid_argument):
        kmeans.init_plusplus(X, 4, dt)
    # the context stays usable afterwards
    assert np.array_equal(kmeans.init_plusplus(X, 2, dt), restated.init_plusplus(X, 2)[0])


@pytest.mark.parametrize("dt", DTYPES)
def test_plusplus_device_memory(dt):
    rng = np.random.default_rng(21)
    X = rng.standard_normal((10000, 24)).astype(dt)
    Xd = torch.from_numpy(X).cuda()
    C = kmeans.init_plusplus(Xd, 50, dt)
    assert C.is_cuda
    assert np.array_equal(C.cpu().numpy(), restated.init_plusplus(X, 50)[0])


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("d", [32, 64])
def test_plusplus_unaligned_device_rows(dt, d):
    """Rows whose start is not 16-byte aligned take the register-staged distance kernel;
    aligned rows take the asynchronous-copy one. Both pick the oracle's rows."""
    rng = np.random.default_rng(41 + d)
    n = 40000
    X = rng.standard_normal((n, d)).astype(dt)
    flat = torch.empty(n * d + 1, dtype=torch.float32 if dt == np.float32 else torch.float64, device="cuda")
    Xd = flat[1:].view(n, d)
    Xd.copy_(torch.from_numpy(X))
    assert Xd.data_ptr() % 16 != 0
    ref = restated.init_plusplus(X, 33)[0]
    assert np.array_equal(kmeans.init_plusplus(Xd, 33, dt).cpu().numpy(), ref)
    assert np.array_equal(kmeans.init_plusplus(torch.from_numpy(X).cuda(), 33, dt).cpu().numpy(), ref)


@pytest.mark.parametrize("dt", DTYPES)
def test_train_without_initial_centroids_smoke(dt):
    """The smoke test, fixture.hpp:221-252: train() with the default k-means++ init on 8
    points, 4 iterations, eps 0.001. The reference compares centroids and responses
    WITHOUT a centroid match, so the init's choice of rows (and hence the order) is pinned:
    centroids (-1.5, -1.5), (1.5, 1.5), responses 1,1,1,1,0,0,0,0, objective 4."""
    X = np.array([1, 1, 2, 2, 1, 2, 2, 1, -1, -1, -1, -2, -2, -1, -2, -2], dt).reshape(8, 2)
    d = kmeans.descriptor(dt).set_cluster_count(2).set_max_iteration_count(4).set_accuracy_threshold(0.001)
    r = kmeans.train(d, X)
    C = r.get_model().get_centroids()
    tol = 5 * np.finfo(dt).eps * r.get_iteration_count() * 100
    assert centroid_rel_err(np.array([[-1.5, -1.5], [1.5, 1.5]]), C) < tol
    assert r.get_responses().ravel().tolist() == [1, 1, 1, 1, 0, 0, 0, 0]
    di = kmeans.descriptor(dt).set_cluster_count(2).set_result_options(
        kmeans.result_options.compute_exact_objective_function)
    inf = kmeans.infer(di, r.get_model(), X)
    assert inf.get_responses().ravel().tolist() == [1, 1, 1, 1, 0, 0, 0, 0]
    assert rel_close(inf.get_objective_function_value(), 4.0, 1e-6)


@pytest.mark.parametrize("dt", DTYPES)
def test_train_default_init_equals_explicit_plusplus_init(dt):
    """train() without initial centroids is train() from kmb_init_plusplus's centers."""
    rng = np.random.default_rng(31)
    X = (rng.standard_normal((30000, 16)) + 5 * rng.integers(0, 8, (30000, 1))).astype(dt)
    d = kmeans.descriptor(dt).set_cluster_count(24).set_max_iteration_count(20).set_accuracy_threshold(0.0)
    a = kmeans.train(d, X)
    C0 = restated.init_plusplus(X, 24)[0]
    b = kmeans.train(d, X, C0)
    assert np.array_equal(a.get_model().get_centroids(), b.get_model().get_centroids())
    assert (a.get_responses() == b.get_responses()).all()
    assert a.get_iteration_count() == b.get_iteration_count()
