"""Generates the golden fixtures in tests/golden/ from the reference project.

Run in a container where the reference tree is mounted:

    python tests/golden/make_golden.py [--reference <reference source tree>]

Sources (paths inside the reference project):

* gold.json -- the "train/infer on gold data" known-answer test:
  cpp/oneapi/dal/algo/kmeans/test/data.hpp:26-184 (100x3 data, k=3 initial and
  expected centroids, expected responses, objective 241.3593613), exercised by
  cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:156-203 (100 iterations, eps 0,
  centroid/objective rel tol 1e-7, responses exact up to centroid matching).
* empty_clusters.json -- "kmeans empty clusters test",
  cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:205-219 (1 iteration).
* smoke_infer.json -- the infer half of the smoke test,
  cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:221-252 (objective 4).
* example_dense.npz -- the k-means example's data and initial centroids
  (data/kmeans_dense_train_data.csv, data/kmeans_dense_train_centroids.csv, used
  by examples/oneapi/cpp/source/kmeans/kmeans_lloyd_dense_batch.cpp with k=20,
  5 iterations, eps 0.001) plus the outputs of the reference DAAL kernel built
  from source (oracle/_ref) on it, in float64 and float32.
* daal_ref_c1.npz -- outputs of the reference kernel on the seeded
  Gaussian-blob workload of the plain CPU configuration at its full size
  (n=100,000, d=20, k=20, init = first k rows, 50 iterations, eps 0), float64
  and float32; daal_ref_c1_small.npz -- the same on its first 20,000 rows, where
  the reference's FP32 trajectory and the restatement's coincide bit for bit.
  Both let the restated oracle and the GPU be re-checked where the reference
  tree is absent.
* daal_ref_plusplus.npz -- the centers chosen by the reference's dense k-means++
  initialisation (DAAL KMeansInitKernel<plusPlusDense>, one trial, mt19937 seeded
  777777: the default of cpp/oneapi/dal/algo/kmeans/detail/train_init_centroids.hpp)
  built from source, float64 and float32, on the seeded inputs of plusplus_cases()
  and on the example data with k=20.
* daal_ref_csr.npz -- outputs of the reference CSR kernels built from source
  (KMeansBatchKernel<lloydCSR>: 25 iterations, eps 0; KMeansInitKernel<plusPlusCSR>)
  on the seeded CSR inputs of csr_cases(), float64 and float32.
* model_archives.npz -- oneDAL binary archives of k-means models written by
  oneDAL's own serialisation code (detail::serialize into binary_output_archive,
  compiled from the reference sources into integration/_build/kmeans_client):
  the model of the serialisation test (cpp/oneapi/dal/algo/kmeans/test/
  serialization.cpp:39-123; trained by the reference kernel with the default
  descriptor and k-means++ init) in float and double with the test rows'
  responses, a 7x3 double model and a model without centroids.
"""
import argparse
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def _numbers(text):
    return [float(v) for v in re.findall(r"-?\d+\.?\d*(?:[eE][-+]?\d+)?", text)]


def _array_after(src, anchor, start=0):
    """Numbers inside the first {...} initializer following `anchor`."""
    i = src.index(anchor, start)
    j = src.index("{", src.index("=", i))
    k = src.index("}", j)
    body = re.sub(r"//[^\n]*", "", src[j + 1:k])
    return _numbers(body), k


def gold(ref):
    src = open(os.path.join(ref, "cpp/oneapi/dal/algo/kmeans/test/data.hpp")).read()
    data, _ = _array_after(src, "get_data()")
    init, _ = _array_after(src, "get_initial_centroids()")
    expc, _ = _array_after(src, "get_expected_centroids()")
    resp, _ = _array_after(src, "get_expected_responses()")
    m = re.search(r"get_expected_objective\(\)\s*{\s*return\s*([0-9.eE+-]+)", src)
    obj = float(m.group(1))
    assert len(data) == 300 and len(init) == 9 and len(expc) == 9 and len(resp) == 100
    return {
        "source": "cpp/oneapi/dal/algo/kmeans/test/data.hpp:26-184; fixture.hpp:156-203",
        "row_count": 100, "column_count": 3, "cluster_count": 3,
        "max_iteration_count": 100, "accuracy_threshold": 0.0,
        "data": data, "initial_centroids": init, "expected_centroids": expc,
        "expected_responses": [int(v) for v in resp], "expected_objective": obj,
        "rel_tol": 1e-7,
    }


def empty_clusters(ref):
    src = open(os.path.join(ref, "cpp/oneapi/dal/algo/kmeans/test/fixture.hpp")).read()
    s = src.index("void check_empty_clusters()")
    data, p = _array_after(src, "data[]", s)
    init, p = _array_after(src, "initial_centroids[]", p)
    fin, p = _array_after(src, "final_centroids[]", p)
    resp, p = _array_after(src, "responses[]", p)
    return {
        "source": "cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:205-219",
        "row_count": 10, "column_count": 1, "cluster_count": 3,
        "max_iteration_count": 1, "accuracy_threshold": 0.0,
        "data": data, "initial_centroids": init, "expected_centroids": fin,
        "expected_responses": [int(v) for v in resp],
    }


def smoke_infer(ref):
    src = open(os.path.join(ref, "cpp/oneapi/dal/algo/kmeans/test/fixture.hpp")).read()
    s = src.index("void check_on_smoke_data()")
    data, p = _array_after(src, "data[]", s)
    fin, p = _array_after(src, "final_centroids[]", p)
    resp, p = _array_after(src, "responses[]", p)
    m = re.search(r"expected_obj_function\s*=\s*([0-9.]+)", src[s:])
    return {
        "source": "cpp/oneapi/dal/algo/kmeans/test/fixture.hpp:221-252 (infer half)",
        "row_count": 8, "column_count": 2, "cluster_count": 2,
        "data": data, "centroids": fin, "expected_responses": [int(v) for v in resp],
        "expected_objective": float(m.group(1)), "rel_tol": 1e-5,
    }


def serialization_case(ref):
    """Train/test rows of the model serialisation test
    (cpp/oneapi/dal/algo/kmeans/test/serialization.cpp:39-72)."""
    src = open(os.path.join(ref, "cpp/oneapi/dal/algo/kmeans/test/serialization.cpp")).read()
    x_test, p = _array_after(src, "x_test[]")
    x_train, p = _array_after(src, "x_train[]", p)
    assert len(x_test) == 20 and len(x_train) == 48
    return np.array(x_train, np.float64).reshape(12, 4), np.array(x_test, np.float64).reshape(5, 4)


def onedal_archive(client, centroids, tag, workdir):
    """oneDAL's own binary archive of a k-means model with `centroids` (k x d; k = 0 for
    a model without centroids), written by the integration client, which runs
    detail::serialize into binary_output_archive compiled from the reference sources."""
    import subprocess
    src = os.path.join(workdir, f"c_{tag}.txt")
    out = os.path.join(workdir, f"m_{tag}.bin")
    k, d = centroids.shape
    with open(src, "w") as f:
        f.write(f"{k} {d}\n" + " ".join(repr(float(v)) for v in centroids.ravel()) + "\n")
    subprocess.run([client, "serialize", src, "double" if centroids.dtype == np.float64 else "float", out],
                   check=True, capture_output=True)
    return np.frombuffer(open(out, "rb").read(), np.uint8)


def csr_cases():
    """Seeded CSR inputs of daal_ref_csr.npz: (name, values, columns, row offsets, d, k,
    initial centroids) -- zero-based, sorted columns, float64."""
    import scipy.sparse as sp
    out = []
    for name, n, d, k, density, seed in (("small", 300, 40, 6, 0.15, 401), ("wide", 2000, 500, 32, 0.02, 402),
                                         ("dense_ish", 800, 24, 12, 0.5, 403)):
        rng = np.random.default_rng(seed)
        M = sp.random(n, d, density=density, format="csr", random_state=seed, dtype=np.float64)
        M.data = rng.standard_normal(M.nnz) * 3
        M.sort_indices()
        C0 = M[rng.choice(n, k, replace=False)].toarray()
        out.append((name, M.data, M.indices.astype(np.int64), M.indptr.astype(np.int64), d, k, C0))
    return out


def blobs_c1(n, seed):
    """Seeded mixture of 20 isotropic Gaussian blobs (std 1) in d=20, centres U[-10,10]."""
    rng = np.random.default_rng(seed)
    k, d = 20, 20
    centres = rng.uniform(-10, 10, size=(k, d))
    lab = rng.integers(0, k, size=n)
    return centres[lab] + rng.standard_normal((n, d))


def plusplus_cases():
    """Seeded inputs of the k-means++ fixtures: (name, X float64, k). Rounded data has
    many duplicate rows, which exercises the reference's resampling."""
    out = []
    for name, n, d, k, seed, kind in (("normal_5k", 5000, 7, 16, 2001, "normal"),
                                      ("blobs_20k", 20000, 20, 20, 2002, "blobs"),
                                      ("ragged_3001", 3001, 33, 100, 2003, "normal"),
                                      ("wide_1500", 1500, 64, 300, 2004, "normal"),
                                      ("dups_4096", 4096, 3, 50, 2005, "rounded")):
        rng = np.random.default_rng(seed)
        if kind == "blobs":
            X = blobs_c1(n, seed)
        else:
            X = 3.0 * rng.standard_normal((n, d))
            if kind == "rounded":
                X = np.round(X)
        out.append((name, X, k))
    return out


def main():
    ap = argparse.ArgumentParser()
    from oracle import build as oracle_build
    ap.add_argument("--reference", default=oracle_build.REFERENCE_TREE)
    ap.add_argument("--only", default=None, choices=["c1"],
                    help="regenerate only these fixtures (c1: daal_ref_c1.npz, daal_ref_c1_small.npz)")
    args = ap.parse_args()
    ref = args.reference

    from oracle import build, daal_ref
    build.build_reference()
    daal_ref.set_threads(1)

    if not args.only:
        for name, fn in (("gold.json", gold), ("empty_clusters.json", empty_clusters), ("smoke_infer.json", smoke_infer)):
            with open(os.path.join(HERE, name), "w") as f:
                json.dump(fn(ref), f, indent=1)

        X = np.loadtxt(os.path.join(ref, "data/kmeans_dense_train_data.csv"), delimiter=",", dtype=np.float64)
        C0 = np.loadtxt(os.path.join(ref, "data/kmeans_dense_train_centroids.csv"), delimiter=",", dtype=np.float64)
        out = {"X": X, "C0": C0}
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            C, lab, obj, it = daal_ref.train(X.astype(dt), C0.astype(dt), 5, 0.001)
            out.update({f"C_{tag}": C, f"labels_{tag}": lab, f"obj_{tag}": obj, f"iters_{tag}": it})
        np.savez_compressed(os.path.join(HERE, "example_dense.npz"), **out)

    # the plain configuration at its full size (n = 100,000 rows, d = 20, k = 20), and a
    # 20,000-row prefix of the same generator on which the FP32 trajectories of the
    # reference and of the restatement coincide bit for bit (at 100,000 rows their
    # different FP32 summation orders move a few near-tie rows, and the trajectories part)
    for fname, n in (("daal_ref_c1.npz", 100_000), ("daal_ref_c1_small.npz", 20_000)):
        X = blobs_c1(n, 1001)
        out = {"seed": 1001, "n": n}
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            Xd = X.astype(dt)
            C, lab, obj, it = daal_ref.train(Xd, Xd[:20].copy(), 50, 0.0)
            out.update({f"C_{tag}": C, f"labels_{tag}": lab.astype(np.uint8), f"obj_{tag}": obj, f"iters_{tag}": it})
        np.savez_compressed(os.path.join(HERE, fname), **out)
    if args.only:
        return

    # k-means++ (train() without initial centroids): the reference's chosen centers
    out = {}
    cases = plusplus_cases() + [("example", np.loadtxt(os.path.join(ref, "data/kmeans_dense_train_data.csv"),
                                                       delimiter=",", dtype=np.float64), 20)]
    for name, X, k in cases:
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            out[f"C_{name}_{tag}"] = daal_ref.init_plusplus(X.astype(dt), k)
    np.savez_compressed(os.path.join(HERE, "daal_ref_plusplus.npz"), **out)

    # CSR Lloyd and plusPlusCSR: outputs of the reference kernels on seeded CSR inputs
    out = {}
    for name, v, c, r, d, k, C0 in csr_cases():
        for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
            daal_ref.set_threads(1)
            C, lab, obj, it = daal_ref.train_csr(v.astype(dt), c, r, d, C0.astype(dt), 25, 0.0)
            out[f"C_{name}_{tag}"], out[f"labels_{name}_{tag}"] = C, lab
            out[f"obj_{name}_{tag}"], out[f"iters_{name}_{tag}"] = obj, it
            out[f"pp_{name}_{tag}"] = daal_ref.init_plusplus_csr(v.astype(dt), c, r, d, k)
    np.savez_compressed(os.path.join(HERE, "daal_ref_csr.npz"), **out)

    # model archives: the serialisation test's model (default descriptor: k = 2, 100
    # iterations, eps 0, k-means++ init) trained by the reference kernel, archived by
    # oneDAL's own serialisation code (integration client), plus the test rows' responses
    client = os.path.join(os.path.dirname(os.path.dirname(HERE)), "integration", "_build", "kmeans_client")
    if os.path.exists(client):
        import tempfile
        x_train, x_test = serialization_case(ref)
        out = {"x_train": x_train, "x_test": x_test}
        with tempfile.TemporaryDirectory() as tmp:
            for dt, tag in ((np.float64, "f64"), (np.float32, "f32")):
                X = x_train.astype(dt)
                C0 = daal_ref.init_plusplus(X, 2)
                C, _, _, _ = daal_ref.train(X, C0, 100, 0.0)
                lab, _ = daal_ref.infer(x_test.astype(dt), C, False)
                out[f"C_{tag}"] = C
                out[f"responses_{tag}"] = lab
                out[f"archive_{tag}"] = onedal_archive(client, C, tag, tmp)
            rng = np.random.default_rng(2024)
            W = rng.standard_normal((7, 3))
            out["C_wide_f64"] = W
            out["archive_wide_f64"] = onedal_archive(client, W, "wide", tmp)
            out["archive_empty"] = onedal_archive(client, np.zeros((0, 0)), "empty", tmp)
        np.savez_compressed(os.path.join(HERE, "model_archives.npz"), **out)
    else:
        print("integration client not built: model_archives.npz left as is")
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
