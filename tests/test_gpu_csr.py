"""GPU tests of kmeans::method::lloyd_csr (kmb_train_csr / kmb_infer_csr) against the
CSR oracle (oracle/kmeans_csr_oracle.c, pinned to the reference CSR kernel) and the
reference suite's CSR cases (cpp/oneapi/dal/algo/kmeans/test/batch.cpp:276-480).

Tolerances: responses exact except rows whose FP64 top-2 score gap lies inside the
working precision's rounding band (the centroid half norms and the sparse products
are summed in a different order than the oracle's); centroids 1e-12 relative per
element (float64) or 1e-5 in Frobenius norm (float32: the float run rounds its
centroids every iteration, which moves near-zero elements by more than 1e-5 of
themselves) and objective 1e-6 relative against the FP64 oracle when every
response matches."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

from helpers import centroid_rel_err, norm_rel_err, rel_close
from onedal_b200 import kmeans
from oracle import restated

pytestmark = pytest.mark.gpu

DTYPES = [np.float64, np.float32]


def _desc(dt, k, T=100, eps=0.0):
    return (kmeans.descriptor(dt, kmeans.method.lloyd_csr).set_cluster_count(k).set_max_iteration_count(T)
            .set_accuracy_threshold(eps))


def _case(seed, n, d, k, density):
    rng = np.random.default_rng(seed)
    M = sp.random(n, d, density=density, format="csr", random_state=seed, dtype=np.float64)
    M.data = rng.standard_normal(M.nnz) * 3
    M.sort_indices()
    C0 = M[rng.choice(n, k, replace=False)].toarray()
    return M, C0


def _band_rows(M, C, dt):
    """Rows whose FP64 top-2 score gap is inside the rounding band of dtype dt."""
    X = M.toarray()
    C = C.astype(np.float64)
    if C.shape[0] < 2:
        return np.zeros(X.shape[0], bool)
    s = 0.5 * (C * C).sum(1)[None, :] - X @ C.T
    part = np.partition(s, 1, axis=1)
    gap = part[:, 1] - part[:, 0]
    u = 2.0 ** -24 if dt == np.float32 else 2.0 ** -53
    xn = np.sqrt((X * X).sum(1))
    cmax = np.sqrt((C * C).sum(1)).max()
    band = 2 * 1.0625 * u * (cmax ** 2 + (X.shape[1] + 2) * xn * cmax)
    return gap <= 4 * band


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("indexing", [kmeans.sparse_indexing.zero_based, kmeans.sparse_indexing.one_based])
def test_csr_exact_objective_accounts_for_unstored_features(dt, indexing):
    """test/batch.cpp:406-480: CSR and dense train agree; objective 100 (the unstored
    features' c^2 terms included)."""
    b = 1 if indexing == kmeans.sparse_indexing.one_based else 0
    t = kmeans.csr_table(np.array([10, 10, 20], dt), np.array([0, 1, 2]) + b, np.array([0, 1, 2, 3]) + b, 3, 3,
                         indexing)
    C0 = np.array([[5, 5, 0], [0, 0, 20]], dt)
    dense = np.array([[10, 0, 0], [0, 10, 0], [0, 0, 20]], dt)
    rc = kmeans.train(_desc(dt, 2, 1).set_result_options(kmeans.result_options.compute_exact_objective_function), t, C0)
    rd = kmeans.train(kmeans.descriptor(dt).set_cluster_count(2).set_max_iteration_count(1), dense, C0)
    assert (rc.get_responses() == rd.get_responses()).all()
    tol = 1e-10 if dt == np.float64 else 1e-5
    assert centroid_rel_err(rd.get_model().get_centroids(), rc.get_model().get_centroids()) < tol
    assert rel_close(rc.get_objective_function_value(), 100.0, tol)
    assert rel_close(rd.get_objective_function_value(), 100.0, tol)
    inf = kmeans.infer(_desc(dt, 2).set_result_options(kmeans.result_options.compute_exact_objective_function),
                       rc.get_model(), t)
    assert rel_close(inf.get_objective_function_value(), 100.0, tol)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("n,d,k,density", [(500, 30, 7, 0.2), (3000, 200, 64, 0.05), (2048, 1000, 130, 0.01),
                                           (5000, 50, 300, 0.3), (1200, 64, 1100, 0.1), (1, 5, 1, 0.5)])
def test_csr_train_matches_oracle(dt, n, d, k, density):
    """Per cluster-chunk shapes (k up to 1024 in one pass, k > 1024 in several), very
    sparse wide rows and near-dense narrow ones, n = 1."""
    M, C0 = _case(n + d + k, n, d, k, density)
    t = kmeans.csr_table.from_scipy(M.astype(dt))
    r = kmeans.train(_desc(dt, k, 30), t, C0.astype(dt))
    Co, lo, oo, ito = restated.train_csr(M.data, M.indices, M.indptr, d, C0, 30, 0.0)
    lab = r.get_responses().ravel()
    near = _band_rows(M, r.get_model().get_centroids(), dt)
    lab_o, _ = restated.infer_csr(M.data, M.indices, M.indptr, d, r.get_model().get_centroids().astype(np.float64),
                                  False)
    assert ((lab == lab_o) | near).all()
    if (lab == lo).all() and r.get_iteration_count() == ito:
        if dt == np.float64:
            assert centroid_rel_err(Co, r.get_model().get_centroids()) < 1e-12
        else:
            assert norm_rel_err(Co, r.get_model().get_centroids()) < 1e-5
        assert rel_close(r.get_objective_function_value(), oo, 1e-6)


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_infer_matches_oracle(dt):
    M, C0 = _case(7, 4000, 300, 50, 0.04)
    t = kmeans.csr_table.from_scipy(M.astype(dt))
    d = _desc(dt, 50).set_result_options(kmeans.result_options.compute_exact_objective_function)
    r = kmeans.infer(d, kmeans.model(C0.astype(dt)), t)
    lo, oo = restated.infer_csr(M.data, M.indices, M.indptr, 300, C0.astype(dt).astype(np.float64), True)
    near = _band_rows(M, C0.astype(dt), dt)
    assert ((r.get_responses().ravel() == lo) | near).all()
    assert rel_close(r.get_objective_function_value(), oo, 1e-6)


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_repeated_runs_are_deterministic(dt):
    """test/batch.cpp:353-404: identical centroids, objective and iteration count."""
    M, C0 = _case(11, 200, 100, 16, 0.05)
    t = kmeans.csr_table.from_scipy(M.astype(dt))
    base = kmeans.train(_desc(dt, 16, 10, 0.01), t, C0.astype(dt))
    for _ in range(4):
        r = kmeans.train(_desc(dt, 16, 10, 0.01), t, C0.astype(dt))
        assert r.get_iteration_count() == base.get_iteration_count()
        assert r.get_objective_function_value() == base.get_objective_function_value()
        assert np.array_equal(r.get_model().get_centroids(), base.get_model().get_centroids())


def _sparse_blobs(n, d, k, seed, dt):
    """Cluster j's rows store values ~ N(5, 0.3) on the columns of column block j
    (disjoint blocks; everything else unstored), so responses are the generating
    cluster ids."""
    rng = np.random.default_rng(seed)
    block = d // k
    rows, cols, vals, truth = [], [], [], rng.integers(0, k, n)
    for i, j in enumerate(truth):
        cc = np.arange(block) + j * block
        rows += [i] * len(cc)
        cols += cc.tolist()
        vals += (5 + 0.3 * rng.standard_normal(len(cc))).tolist()
    M = sp.csr_matrix((np.array(vals, dt), (np.array(rows), np.array(cols))), shape=(n, d))
    M.sort_indices()
    return M, truth


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("k,n,d", [(5, 50, 20), (16, 200, 100), (128, 20000, 1024)])
def test_csr_sparse_blobs_with_initial_centroids(dt, k, n, d):
    """test/batch.cpp:276-351 ('sparse default cases', with initial centroids): responses
    equal the generating clusters."""
    M, truth = _sparse_blobs(n, d, k, 3 + k, dt)
    first = np.array([np.flatnonzero(truth == j)[0] for j in range(k)])
    C0 = M[first].toarray()
    r = kmeans.train(_desc(dt, k, 10, 0.01), kmeans.csr_table.from_scipy(M), C0)
    assert (r.get_responses().ravel() == truth).all()


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_device_tensors_and_index_bases_agree(dt):
    M, C0 = _case(5, 3000, 120, 20, 0.08)
    M = M.astype(dt)
    host = kmeans.train(_desc(dt, 20, 15), kmeans.csr_table.from_scipy(M), C0.astype(dt))
    tdt = torch.float32 if dt == np.float32 else torch.float64
    for base in (0, 1):
        t = kmeans.csr_table(torch.from_numpy(M.data).cuda(), torch.from_numpy(M.indices.astype(np.int64) + base).cuda(),
                             torch.from_numpy(M.indptr.astype(np.int64) + base).cuda(), 3000, 120, base)
        r = kmeans.train(_desc(dt, 20, 15), t, torch.from_numpy(C0.astype(dt)).cuda())
        assert r.get_model().get_centroids().dtype == tdt
        assert np.array_equal(r.get_model().get_centroids().cpu().numpy(), host.get_model().get_centroids())
        assert np.array_equal(r.get_responses().cpu().numpy().ravel(), host.get_responses().ravel())


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_empty_clusters_are_reseeded_like_oracle(dt):
    M, C0 = _case(42, 300, 40, 12, 0.1)
    C0[5:] = C0[0]
    r = kmeans.train(_desc(dt, 12, 10), kmeans.csr_table.from_scipy(M.astype(dt)), C0.astype(dt))
    Co, lo, oo, ito = restated.train_csr(M.data, M.indices, M.indptr, 40, C0, 10, 0.0)
    assert r.stats.empty_cluster_events > 0
    if dt == np.float64:
        assert (r.get_responses().ravel() == lo).all() and r.get_iteration_count() == ito
        assert centroid_rel_err(Co, r.get_model().get_centroids()) < 1e-12


def test_csr_malformed_input_is_invalid_argument():
    good_v, good_c, good_r = np.array([1.0, 2.0, 3.0]), np.array([0, 2, 1]), np.array([0, 2, 3])
    C0 = np.zeros((1, 3))
    for c, r in ((np.array([2, 0, 1]), good_r),      # not increasing within row 0
                 (np.array([0, 0, 1]), good_r),      # duplicate column
                 (np.array([0, 3, 1]), good_r),      # column out of range
                 (good_c, np.array([0, 3, 2])),      # decreasing offsets
                 (good_c, np.array([1, 2, 3]))):     # offsets not starting at the base
        t = kmeans.csr_table(good_v, c, r, 2, 3, kmeans.sparse_indexing.zero_based)
        with pytest.raises(kmeans.invalid_argument):
            kmeans.train(_desc(np.float64, 1, 2), t, C0)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("n,d,k,density", [(1, 4, 1, 0.5), (513, 40, 17, 0.1), (5000, 300, 64, 0.03),
                                           (70001, 2000, 40, 0.005)])
def test_csr_plusplus_matches_oracle(dt, n, d, k, density):
    """plusPlusCSR on the GPU picks the oracle's rows exactly (the oracle is pinned to the
    reference build): ragged block counts, empty rows, wide sparse rows."""
    M, _ = _case(n + k, n, d, 1, density)
    M = M.astype(dt)
    C = kmeans.init_plusplus_csr(kmeans.csr_table.from_scipy(M), k, dt)
    Co, rows = restated.init_plusplus_csr(M.data, M.indices.astype(np.int64), M.indptr.astype(np.int64), d, k)
    assert np.array_equal(C, Co)


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_plusplus_device_rows_and_pool_refill(dt, monkeypatch):
    M, _ = _case(17, 4000, 150, 1, 0.05)
    M = M.astype(dt)
    M.data = np.round(M.data).astype(dt) + dt(0.5)  # duplicate-heavy: resampling happens
    ref = restated.init_plusplus_csr(M.data, M.indices.astype(np.int64), M.indptr.astype(np.int64), 150, 30)[0]
    monkeypatch.setenv("KMB_PLUSPLUS_POOL", "1")
    assert np.array_equal(kmeans.init_plusplus_csr(kmeans.csr_table.from_scipy(M), 30, dt), ref)
    t = kmeans.csr_table(torch.from_numpy(M.data).cuda(), torch.from_numpy(M.indices.astype(np.int64) + 1).cuda(),
                         torch.from_numpy(M.indptr.astype(np.int64) + 1).cuda(), 4000, 150,
                         kmeans.sparse_indexing.one_based)
    assert np.array_equal(kmeans.init_plusplus_csr(t, 30, dt).cpu().numpy(), ref)


@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("k,n,d", [(5, 50, 20), (16, 200, 100), (32, 10000, 512)])
def test_csr_sparse_blobs_without_initial_centroids(dt, k, n, d):
    """test/batch.cpp:276-351 without initial centroids: the default plusPlusCSR init.
    The responses are the oracle's from the oracle's k-means++ centers (the same rows the
    reference build picks); with float32 draws on the (16, 200, 100) case the reference
    itself places two centers in one generating cluster, so the recovered partition is
    checked against the oracle rather than the generator."""
    M, truth = _sparse_blobs(n, d, k, 5 + k, dt)
    r = kmeans.train(_desc(dt, k, 30, 0.01), kmeans.csr_table.from_scipy(M))
    C0 = restated.init_plusplus_csr(M.data, M.indices.astype(np.int64), M.indptr.astype(np.int64), d, k)[0]
    r2 = kmeans.train(_desc(dt, k, 30, 0.01), kmeans.csr_table.from_scipy(M), C0)
    assert np.array_equal(r.get_model().get_centroids(), r2.get_model().get_centroids())
    _, lo, _, ito = restated.train_csr(M.data, M.indices, M.indptr, d, C0, 30, 0.01)
    assert (r.get_responses().ravel() == lo).all() and r.get_iteration_count() == ito


@pytest.mark.parametrize("k,n,d", [(16, 20000, 160), (128, 20000, 1024)])
def test_csr_float_centroids_equal_dense_bit_for_bit(k, n, d):
    """Float values: the CSR update sums the stored entries as the same exact integers
    as the dense rows' update (column scales from the largest |x|, an unstored entry
    adds zero), so with equal responses the centroids are the same floats, bit for
    bit, in full passes and in passes that apply only the moved rows."""
    M, truth = _sparse_blobs(n, d, k, 11 + k, np.float32)
    first = np.array([np.flatnonzero(truth == j)[0] for j in range(k)])
    C0 = M[first].toarray()
    rc = kmeans.train(_desc(np.float32, k, 6), kmeans.csr_table.from_scipy(M), C0)
    rd = kmeans.train(kmeans.descriptor(np.float32).set_cluster_count(k).set_max_iteration_count(6)
                      .set_accuracy_threshold(0.0), M.toarray(), C0)
    assert (rc.get_responses() == rd.get_responses()).all()
    assert rc.get_iteration_count() == rd.get_iteration_count()
    assert np.array_equal(rc.get_model().get_centroids(), rd.get_model().get_centroids())
