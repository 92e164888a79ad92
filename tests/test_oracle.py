"""CPU tests: the oracle is pinned against the reference's golden vectors and
against the reference's own DAAL kernel compiled from source."""
import numpy as np
import pytest

from helpers import centroid_rel_err, find_match_centroids, load_json, rel_close
from oracle import daal_ref, restated

DTYPES = [np.float64, np.float32]


@pytest.mark.parametrize("dt", DTYPES)
def test_gold_known_answer(dt):
    """cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:156-203 with data.hpp:26-184."""
    g = load_json("gold.json")
    X = np.array(g["data"], dt).reshape(100, 3)
    C0 = np.array(g["initial_centroids"], dt).reshape(3, 3)
    C, lab, obj, it = restated.train(X, C0, g["max_iteration_count"], g["accuracy_threshold"])
    exp = np.array(g["expected_centroids"]).reshape(3, 3)
    m = find_match_centroids(exp, C)
    tol = 1e-7 if dt == np.float64 else 1e-6
    assert centroid_rel_err(exp, C, m) < tol
    assert rel_close(obj, g["expected_objective"], tol)
    # responses under the centroid permutation (fixture.hpp:191-193)
    assert (m[lab] == np.array(g["expected_responses"])).all()


@pytest.mark.parametrize("dt", DTYPES)
def test_empty_clusters_known_answer(dt):
    """'kmeans empty clusters test', fixture.hpp:205-219: reseed order and responses."""
    e = load_json("empty_clusters.json")
    X = np.array(e["data"], dt).reshape(10, 1)
    C0 = np.array(e["initial_centroids"], dt).reshape(3, 1)
    C, lab, obj, it = restated.train(X, C0, 1, 0.0)
    np.testing.assert_allclose(C.ravel(), e["expected_centroids"], rtol=5 * np.finfo(dt).eps * 100)
    assert lab.tolist() == e["expected_responses"]
    assert it == 1


@pytest.mark.parametrize("dt", DTYPES)
def test_smoke_infer_known_answer(dt):
    """Infer half of the smoke test, fixture.hpp:221-252: objective 4."""
    s = load_json("smoke_infer.json")
    X = np.array(s["data"], dt).reshape(8, 2)
    C = np.array(s["centroids"], dt).reshape(2, 2)
    lab, obj = restated.infer(X, C, True)
    assert lab.tolist() == s["expected_responses"]
    assert rel_close(obj, s["expected_objective"], s["rel_tol"])


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_example_dataset_matches_reference_kernel(tag, dt):
    """The k-means example's data (data/kmeans_dense_train_*.csv, k=20, 5 iterations,
    eps 0.001) against outputs of the reference kernel recorded in the fixture."""
    z = np.load(__import__("os").path.join(__import__("helpers").GOLDEN, "example_dense.npz"))
    C, lab, obj, it = restated.train(z["X"].astype(dt), z["C0"].astype(dt), 5, 0.001)
    assert it == int(z[f"iters_{tag}"])
    assert (lab == z[f"labels_{tag}"]).all()
    assert centroid_rel_err(z[f"C_{tag}"], C) < (1e-13 if dt == np.float64 else 1e-6)
    assert rel_close(obj, float(z[f"obj_{tag}"]), 1e-12 if dt == np.float64 else 1e-6)


@pytest.mark.parametrize("fixture", ["daal_ref_c1.npz", "daal_ref_c1_small.npz"])
@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_blob_workload_matches_reference_kernel(tag, dt, fixture):
    """The plain configuration (d=20, k=20, init = first rows, eps 0, 50 max
    iterations) at its full 100,000 rows and on a 20,000-row prefix, against recorded
    reference-kernel outputs. float64 matches bit for bit at both sizes; float32
    too on the prefix. At 100,000 rows the two FP32 summation orders (the
    reference's per-thread partials and BLAS blocking, the restatement's row order)
    move a few near-tie rows and the unconverged trajectories part, so there float32
    is held to the iteration count, 0.5 % of the labels and the objective to 1e-5."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import blobs_c1
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", fixture))
    X = blobs_c1(int(z["n"]), int(z["seed"])).astype(dt)
    C, lab, obj, it = restated.train(X, X[:20].copy(), 50, 0.0)
    assert it == int(z[f"iters_{tag}"])
    if dt == np.float32 and int(z["n"]) > 20000:
        assert (lab != z[f"labels_{tag}"]).mean() < 5e-3
        assert rel_close(obj, float(z[f"obj_{tag}"]), 1e-5)
        return
    assert (lab == z[f"labels_{tag}"]).all()
    assert centroid_rel_err(z[f"C_{tag}"], C) < (1e-13 if dt == np.float64 else 1e-6)
    assert rel_close(obj, float(z[f"obj_{tag}"]), 1e-12 if dt == np.float64 else 1e-6)


needs_ref = pytest.mark.skipif(not daal_ref.available(), reason="reference kernel not built (make -C oracle/ref)")


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("n,d,k", [(257, 3, 5), (1000, 7, 31), (513, 33, 130), (64, 2, 64)])
def test_restated_equals_reference_kernel_f64(seed, n, d, k):
    """Live comparison with the reference DAAL kernel (single thread), ragged shapes,
    including k == n (every row its own cluster) and empty-cluster reseeding."""
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, d)) * rng.uniform(0.5, 3.0, d)
    C0 = X[rng.choice(n, k, replace=False)].copy() if seed != 2 else np.repeat(X[:1], k, axis=0) + 1e-3 * np.arange(k)[:, None]
    daal_ref.set_threads(1)
    r = daal_ref.train(X, C0, 30, 0.0)
    s = restated.train(X, C0, 30, 0.0)
    assert s[3] == r[3]
    assert (s[1] == r[1]).all()
    assert centroid_rel_err(r[0], s[0]) < 1e-12
    assert rel_close(s[2], r[2], 1e-12)


@needs_ref
def test_reference_kernel_thread_count_does_not_change_f64_labels():
    rng = np.random.default_rng(5)
    X = rng.standard_normal((5000, 8))
    C0 = X[:16].copy()
    daal_ref.set_threads(1)
    a = daal_ref.train(X, C0, 10, 0.0)
    daal_ref.set_threads(4)
    b = daal_ref.train(X, C0, 10, 0.0)
    daal_ref.set_threads(1)
    assert (a[1] == b[1]).all() and a[3] == b[3]
    assert centroid_rel_err(a[0], b[0]) < 1e-12


def test_step_matches_train_first_iteration():
    rng = np.random.default_rng(3)
    X = rng.standard_normal((600, 5))
    C0 = X[:7].copy()
    C1, lab, shift, ne, goal = restated.step(X, C0)
    C, _, _, it = restated.train(X, C0, 1, 0.0)
    assert it == 1
    np.testing.assert_array_equal(C, C1)
    assert shift > 0 and ne == 0


def test_planted_label_flip_is_detected():
    """A mistake planted in the oracle's output (one flipped label, one perturbed
    centroid) must fail the same checks the GPU parity tests apply."""
    g = load_json("gold.json")
    X = np.array(g["data"]).reshape(100, 3)
    C0 = np.array(g["initial_centroids"]).reshape(3, 3)
    C, lab, obj, it = restated.train(X, C0, 100, 0.0)
    bad = lab.copy()
    bad[17] = (bad[17] + 1) % 3
    m = find_match_centroids(np.array(g["expected_centroids"]).reshape(3, 3), C)
    assert not (m[bad] == np.array(g["expected_responses"])).all()
    Cb = C.copy()
    Cb[1, 2] *= 1 + 1e-5
    assert centroid_rel_err(C, Cb) > 1e-7


def _plusplus_inputs():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import plusplus_cases
    from helpers import GOLDEN
    z = np.load(os.path.join(GOLDEN, "example_dense.npz"))
    return plusplus_cases() + [("example", z["X"], 20)]


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_plusplus_matches_reference_fixtures(tag, dt):
    """The restated k-means++ picks exactly the reference's centers (bit-identical rows of
    X), duplicate-heavy data included, in both precisions."""
    import os
    from helpers import GOLDEN
    z = np.load(os.path.join(GOLDEN, "daal_ref_plusplus.npz"))
    for name, X, k in _plusplus_inputs():
        X = X.astype(dt)
        C, rows = restated.init_plusplus(X, k)
        assert C.dtype == dt
        assert np.array_equal(C, z[f"C_{name}_{tag}"]), name
        assert np.array_equal(C, X[rows]), name
        assert (rows >= 0).all() and (rows < len(X)).all()


def test_plusplus_fused_and_unfused_distance_agree_on_fixtures():
    """The oracle's distance loop with and without FMA contraction picks the same rows on
    the fixture data (the reference build is compiled with contraction)."""
    for name, X, k in _plusplus_inputs()[:3]:
        a = restated.init_plusplus(X, k)[1]
        b = restated.init_plusplus(X, k, fused=False)[1]
        assert (a == b).all(), name


@needs_ref
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("n,d,k,seed", [(1, 1, 1, 0), (7, 2, 7, 1), (513, 5, 40, 2), (1025, 9, 3, 3), (2000, 1, 3, 4),
                                         (3000, 2, 9, 5)])
def test_plusplus_restated_equals_reference_live(dt, n, d, k, seed):
    """Live comparison with the reference build on ragged shapes: n not a multiple of the
    512-row block, k == n, d == 1, and tiny integer grids with exactly k distinct rows
    (many duplicates, so the reference resamples candidates within its epsilon)."""
    rng = np.random.default_rng(seed)
    X = rng.integers(0, 3, (n, d)).astype(dt) if seed >= 4 else rng.standard_normal((n, d)).astype(dt)
    for s in (777777, 12345):
        assert np.array_equal(restated.init_plusplus(X, k, s)[0], daal_ref.init_plusplus(X, k, s))


@pytest.mark.parametrize("dt", DTYPES)
def test_plusplus_fewer_distinct_rows_than_k_is_an_error(dt):
    """With fewer than k distinct rows every distance becomes zero and the reference's
    resampling loop (kmeans_plusplus_init_impl.i:613-635) never ends; the restatement
    reports it instead (the reference build is not run on this input)."""
    X = np.repeat(np.arange(3, dtype=dt)[:, None], 100, axis=0)
    assert len(restated.init_plusplus(X, 3)[1]) == 3
    with pytest.raises(restated.NoCandidateRows):
        restated.init_plusplus(X, 4)


@pytest.mark.parametrize("dt", DTYPES)
def test_plusplus_smoke_known_answer(dt):
    """fixture.hpp:221-252 trains the 8-point smoke data without initial centroids and
    compares centroids and responses without a centroid match: the k-means++ rows picked
    with seed 777777 fix the order (-1.5, -1.5), (1.5, 1.5) and responses 1,1,1,1,0,0,0,0."""
    X = np.array([1, 1, 2, 2, 1, 2, 2, 1, -1, -1, -1, -2, -2, -1, -2, -2], dt).reshape(8, 2)
    C0, rows = restated.init_plusplus(X, 2)
    C, lab, obj, it = restated.train(X, C0, 4, 0.001)
    assert centroid_rel_err(np.array([[-1.5, -1.5], [1.5, 1.5]]), C) < 5 * np.finfo(dt).eps * it * 100
    assert lab.tolist() == [1, 1, 1, 1, 0, 0, 0, 0]
    assert rel_close(obj, 4.0, 1e-6)


def _sparse_case(seed, n, d, k, density, dt):
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    M = sp.random(n, d, density=density, format="csr", random_state=seed, dtype=np.float64)
    M.data = rng.standard_normal(M.nnz) * 3
    M.sort_indices()
    C0 = M[rng.choice(n, k, replace=False)].toarray()
    return M.data.astype(dt), M.indices.astype(np.int64), M.indptr.astype(np.int64), C0.astype(dt)


def test_csr_exact_objective_known_answer():
    """'KMeans CSR exact objective accounts for unstored features' (test/batch.cpp:406-480):
    3 rows with one stored value each, 2 centroids, 1 iteration: the CSR objective equals
    the dense one (100), the responses and centroids too."""
    v = np.array([10, 10, 20.0])
    c = np.array([0, 1, 2])
    r = np.array([0, 1, 2, 3])
    C0 = np.array([[5, 5, 0], [0, 0, 20.0]])
    dense = np.array([[10, 0, 0], [0, 10, 0], [0, 0, 20.0]])
    for dt in DTYPES:
        Cs, ls, os_, its = restated.train_csr(v.astype(dt), c, r, 3, C0.astype(dt), 1, 0.0)
        Cd, ld, od, itd = restated.train(dense.astype(dt), C0.astype(dt), 1, 0.0)
        assert (ls == ld).all() and its == itd == 1
        assert centroid_rel_err(Cd, Cs) < (1e-10 if dt == np.float64 else 1e-5)
        assert rel_close(os_, 100.0, 1e-6) and rel_close(od, 100.0, 1e-6)


@needs_ref
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("seed", range(6))
def test_csr_restated_equals_reference_kernel(seed, dt):
    """Live comparison with the reference KMeansBatchKernel<lloydCSR> (single thread):
    responses and iteration count exact, centroids and objective to rounding."""
    rng = np.random.default_rng(100 + seed)
    n, d, k = int(rng.integers(30, 700)), int(rng.integers(4, 150)), int(rng.integers(2, 30))
    v, c, r, C0 = _sparse_case(seed, n, d, k, float(rng.uniform(0.03, 0.3)), dt)
    daal_ref.set_threads(1)
    a = restated.train_csr(v, c, r, d, C0, 25, 0.0)
    b = daal_ref.train_csr(v, c, r, d, C0, 25, 0.0)
    assert (a[1] == b[1]).all() and a[3] == b[3]
    tol = 1e-12 if dt == np.float64 else 1e-5
    assert centroid_rel_err(b[0], a[0]) < tol
    assert rel_close(a[2], b[2], tol)
    la, oa = restated.infer_csr(v, c, r, d, a[0], True)
    lb, ob = daal_ref.infer_csr(v, c, r, d, a[0], True)
    assert (la == lb).all() and rel_close(oa, ob, tol)


@needs_ref
def test_csr_reference_reseeds_empty_clusters_like_restatement():
    """Duplicate initial centroids force empty clusters; the reseeded centers (farthest
    rows expanded to dense) agree."""
    v, c, r, C0 = _sparse_case(42, 300, 40, 12, 0.1, np.float64)
    C0[5:] = C0[0]
    daal_ref.set_threads(1)
    a = restated.train_csr(v, c, r, 40, C0, 10, 0.0)
    b = daal_ref.train_csr(v, c, r, 40, C0, 10, 0.0)
    assert (a[1] == b[1]).all() and a[3] == b[3]
    assert centroid_rel_err(b[0], a[0]) < 1e-12


@needs_ref
@pytest.mark.parametrize("dt", DTYPES)
@pytest.mark.parametrize("seed", range(8))
def test_plusplus_csr_restated_equals_reference_live(seed, dt):
    """plusPlusCSR (the lloyd_csr default init): the restatement picks the reference
    build's centers exactly, including rounded values (duplicate rows) and empty rows."""
    import scipy.sparse as sp
    rng = np.random.default_rng(300 + seed)
    n, d = int(rng.integers(10, 2500)), int(rng.integers(3, 250))
    k = min(int(rng.integers(1, 50)), n)
    M = sp.random(n, d, density=float(rng.uniform(0.02, 0.4)), format="csr", random_state=seed)
    M.data = rng.standard_normal(M.nnz) * 2
    if seed % 3 == 0:
        M.data = np.round(M.data) + 0.5
    M.sort_indices()
    v = M.data.astype(dt)
    a, rows = restated.init_plusplus_csr(v, M.indices, M.indptr, d, k)
    b = daal_ref.init_plusplus_csr(v, M.indices, M.indptr, d, k)
    assert np.array_equal(a, b)
    assert np.array_equal(a, M[rows].toarray().astype(dt))


@pytest.mark.parametrize("tag,dt", [("f64", np.float64), ("f32", np.float32)])
def test_csr_restated_matches_reference_fixtures(tag, dt):
    """The CSR restatement against the reference CSR kernels' recorded outputs
    (tests/golden/daal_ref_csr.npz), usable where the reference build is absent."""
    import os
    import sys
    from helpers import GOLDEN
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    from make_golden import csr_cases
    z = np.load(os.path.join(GOLDEN, "daal_ref_csr.npz"))
    for name, v, c, r, d, k, C0 in csr_cases():
        C, lab, obj, it = restated.train_csr(v.astype(dt), c, r, d, C0.astype(dt), 25, 0.0)
        assert (lab == z[f"labels_{name}_{tag}"]).all() and it == int(z[f"iters_{name}_{tag}"]), name
        tol = 1e-12 if dt == np.float64 else 1e-5
        assert centroid_rel_err(z[f"C_{name}_{tag}"], C) < tol, name
        assert rel_close(obj, float(z[f"obj_{name}_{tag}"]), tol), name
        assert np.array_equal(restated.init_plusplus_csr(v.astype(dt), c, r, d, k)[0], z[f"pp_{name}_{tag}"]), name


def test_cluster_stats_checker_matches_numpy():
    """The full-size tests' host checker (FP64 sums, counts and objective of given
    labels, threaded) against a plain numpy evaluation."""
    rng = np.random.default_rng(5)
    n, d, k = 30011, 13, 41
    X = rng.standard_normal((n, d)).astype(np.float32) * 4
    lab = rng.integers(0, k - 1, n).astype(np.int32)  # cluster k-1 stays empty
    C = rng.standard_normal((k, d)).astype(np.float32)
    sums, counts, obj = restated.cluster_stats_f32(X, lab, k, C)
    ref = np.zeros((k, d))
    np.add.at(ref, lab, X.astype(np.float64))
    np.testing.assert_allclose(sums, ref, rtol=1e-12, atol=1e-9)
    np.testing.assert_array_equal(counts, np.bincount(lab, minlength=k))
    assert counts[-1] == 0
    o = ((X.astype(np.float64) - C[lab].astype(np.float64)) ** 2).sum()
    assert abs(obj - o) <= 1e-12 * o
    with pytest.raises(restated.OracleError):
        restated.cluster_stats_f32(X, np.full(n, k, np.int32), k)
