"""CPU tests (gloo, world size 2 and 3) of the row-sharded Lloyd exchange in
onedal_b200.spmd: all-reduce of FP64 sums/counts, identical finalize on every
rank, global empty-cluster reseeding, convergence. The per-rank compute is a
numpy stand-in with the same contract as DeviceShardOps; the result must equal
the single-process FP64 oracle run (responses, iteration count, centroids,
objective) and be identical on all ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from onedal_b200.spmd import ShardStats, train_spmd


class NumpyShardOps:
    """CPU stand-in for DeviceShardOps (float64)."""

    def __init__(self, X):
        self.X = torch.from_numpy(np.ascontiguousarray(X, np.float64))

    def partial(self, C):
        X = self.X.numpy()
        Cn = C.numpy()
        h = 0.5 * (Cn * Cn).sum(1)
        score = h[None, :] - X @ Cn.T
        lab = score.argmin(1).astype(np.int32)
        best = score[np.arange(X.shape[0]), lab]
        k, d = Cn.shape
        sums = np.zeros((k, d))
        np.add.at(sums, lab, X)
        counts = np.bincount(lab, minlength=k).astype(np.int64)
        row_sq = 2.0 * best + (X * X).sum(1)
        return ShardStats(torch.from_numpy(lab), torch.from_numpy(sums), torch.from_numpy(counts),
                          torch.from_numpy(row_sq), float(((X - Cn[lab]) ** 2).sum()))

    def finalize(self, sums, counts, C):
        S, n, Cn = sums.numpy(), counts.numpy(), C.numpy()
        out = Cn.copy()
        nz = n > 0
        out[nz] = S[nz] / n[nz, None]
        shift = float(((Cn[nz] - out[nz]) ** 2).sum())
        return torch.from_numpy(out), shift, [int(i) for i in np.nonzero(~nz)[0]]

    def rows(self, idx):
        return self.X[idx.to(torch.long)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, X, C0, T, eps, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        bounds = np.linspace(0, X.shape[0], world + 1).astype(int)
        ops = NumpyShardOps(X[bounds[rank]:bounds[rank + 1]])
        C, lab, it, obj = train_spmd(ops, torch.from_numpy(C0.copy()), T, eps)
        out_q.put((rank, C.numpy(), lab.numpy(), it, obj))
    finally:
        dist.destroy_process_group()


def _run(world, X, C0, T, eps):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, X, C0, T, eps, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(res, key=lambda r: r[0])


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_train_equals_single_process_oracle(world):
    from oracle import restated
    rng = np.random.default_rng(41)
    centres = rng.uniform(-10, 10, (12, 6))
    X = centres[rng.integers(0, 12, 3001)] + rng.standard_normal((3001, 6))
    C0 = X[:12].copy()
    res = _run(world, X, C0, 50, 0.0)
    ref_C, ref_lab, ref_obj, ref_it = restated.train(X, C0, 50, 0.0)
    for r in res:  # identical centroids on every rank
        np.testing.assert_array_equal(r[1], res[0][1])
        assert r[3] == ref_it
    np.testing.assert_allclose(res[0][1], ref_C, rtol=1e-12, atol=1e-12)
    assert (np.concatenate([r[2] for r in res]) == ref_lab).all()
    assert abs(res[0][4] - ref_obj) <= 1e-9 * ref_obj


def test_sharded_empty_cluster_reseed_matches_oracle():
    """Duplicate initial centroids force empty clusters; the global farthest rows must
    reseed them in ascending cluster order on every rank."""
    from oracle import restated
    rng = np.random.default_rng(42)
    X = rng.standard_normal((1200, 4)) * rng.uniform(0.5, 3, 4)
    C0 = np.repeat(X[:1], 6, axis=0) + 1e-3 * np.arange(6)[:, None]
    res = _run(2, X, C0, 5, 0.0)
    ref_C, ref_lab, ref_obj, ref_it = restated.train(X, C0, 5, 0.0)
    np.testing.assert_array_equal(res[0][1], res[1][1])
    np.testing.assert_allclose(res[0][1], ref_C, rtol=1e-12, atol=1e-12)
    assert (np.concatenate([r[2] for r in res]) == ref_lab).all()
    assert res[0][3] == ref_it
