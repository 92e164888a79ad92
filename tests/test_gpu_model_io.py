"""GPU side of model serialisation: the reference's serialisation test
(cpp/oneapi/dal/algo/kmeans/test/serialization.cpp:98-123) through this path, and
device-resident centroids moving through archives (device -> archive -> device, and
straight into the serving engine's resident model store)."""
import os

import numpy as np
import pytest
import torch

from helpers import GOLDEN
from onedal_b200 import kmeans, serving

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,dt", [("f32", np.float32), ("f64", np.float64)])
def test_reference_serialization_test(tag, dt):
    """Train with the default descriptor (k = 2, 100 iterations, eps 0, k-means++ init),
    serialise, deserialise, infer on the test rows with both models: equal responses.
    The trained centroids match the reference kernel's model recorded in the fixture,
    and the test rows' responses are the reference's."""
    z = np.load(os.path.join(GOLDEN, "model_archives.npz"))
    desc = kmeans.descriptor(dt)
    m = kmeans.train(desc, z["x_train"].astype(dt)).get_model()
    m2 = kmeans.model.deserialize(m.serialize())
    a = kmeans.infer(desc, m, z["x_test"].astype(dt)).get_responses().ravel()
    b = kmeans.infer(desc, m2, z["x_test"].astype(dt)).get_responses().ravel()
    assert (a == b).all()
    tol = 1e-6 if dt == np.float32 else 1e-12
    assert np.allclose(m.get_centroids(), z[f"C_{tag}"], rtol=tol, atol=tol)
    assert (a == z[f"responses_{tag}"]).all()


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_device_resident_round_trip(dt):
    rng = np.random.default_rng(5)
    C = rng.standard_normal((300, 96)).astype(dt)
    Cd = torch.from_numpy(C).cuda()
    archive = kmeans.model(Cd).serialize()
    assert archive == kmeans.model(C).serialize()
    m = kmeans.model.deserialize(archive, device="cuda")
    assert m.get_centroids().is_cuda
    assert torch.equal(m.get_centroids(), Cd)
    X = torch.from_numpy(rng.standard_normal((5000, 96)).astype(dt)).cuda()
    desc = kmeans.descriptor(dt).set_cluster_count(300)
    r1 = kmeans.infer(desc, m, X).get_responses()
    r2 = kmeans.infer(desc, kmeans.model(C), X.cpu().numpy()).get_responses()
    assert np.array_equal(r1.cpu().numpy().ravel(), np.asarray(r2).ravel())


def test_server_loads_archives():
    rng = np.random.default_rng(9)
    C = rng.standard_normal((64, 24)).astype(np.float32)
    X = rng.standard_normal((4000, 24)).astype(np.float32)
    expect = np.asarray(kmeans.infer(kmeans.descriptor(np.float32).set_cluster_count(64), kmeans.model(C), X)
                        .get_responses()).ravel()
    srv = serving.KMeansServer(0, hbm_budget_bytes=4 << 30, lanes=1, trainers=1)
    try:
        mid = srv.add_model_serialized(kmeans.model(C).serialize())
        req = srv.submit_infer(mid, X)
        labels, _ = srv.wait(req)
        assert (labels == expect).all()
        with pytest.raises(serving.ServingError):
            srv.add_model_serialized(b"not an archive")
        with pytest.raises(serving.ServingError):
            srv.add_model_serialized(kmeans.model().serialize())  # no centroids to serve
    finally:
        srv.close()
