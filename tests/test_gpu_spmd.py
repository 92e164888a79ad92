"""GPU side of the row-sharded Lloyd path (onedal_b200.spmd.DeviceShardOps over
kmb_partial_sums / kmb_finalize_centroids), in one process on one GPU:

- shards of one matrix give per-shard FP64 sums and counts whose sum, finalized on
  the device, is the FP64 oracle's single-process update (responses, centroids,
  shift, empty clusters), with widths that take several 128-column tiles;
- train_spmd over a one-rank NCCL group equals the oracle's training run
  (responses, iteration count, centroids, objective), an emptied cluster included.

The exchange itself with two and three ranks is covered on the CPU (gloo) with the
same train_spmd code."""
import datetime
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from helpers import centroid_rel_err, rel_close
from onedal_b200 import _native
from onedal_b200.spmd import DeviceShardOps, train_spmd
from oracle import restated

pytestmark = pytest.mark.gpu

CENTROID_TOL = {np.float32: 1e-6, np.float64: 1e-12}


def _blobs(n, d, k, dt, seed, far_centroid=False):
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-20, 20, (k, d))
    lab = rng.integers(0, k, n)
    X = (centers[lab] + rng.standard_normal((n, d))).astype(dt)
    # one start near each blob's center: no row lies near a bisector, so float32
    # responses equal the FP64 oracle's
    C0 = (centers + 0.1 * rng.standard_normal((k, d))).astype(dt)
    if far_centroid:
        C0[k // 2] = 1e4  # nearest to no row: its cluster is empty after the first assignment
    return X, C0


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("d,k,far", [(300, 37, False), (130, 129, True), (20, 5, False)])
def test_shard_sums_match_single_update(dt, d, k, far):
    n = 20000
    X, C0 = _blobs(n, d, k, dt, seed=d + k, far_centroid=far)
    Cd = torch.from_numpy(C0).cuda()
    cuts = [0, 7001, 12000, n]
    sums = torch.zeros((k, d), dtype=torch.float64, device="cuda")
    counts = torch.zeros(k, dtype=torch.int64, device="cuda")
    labels = []
    sq = 0.0
    ops = None
    for a, b in zip(cuts[:-1], cuts[1:]):
        ops = DeviceShardOps(torch.from_numpy(X[a:b]).cuda())
        st = ops.partial(Cd)
        sums += st.sums
        counts += st.counts
        labels.append(st.labels.cpu().numpy())
        sq += float(st.sq_total)
    C_new, shift, empty = ops.finalize(sums, counts, Cd)
    torch.cuda.synchronize()

    C64, lab64, shift64, ne64, _ = restated.step(X.astype(np.float64), C0.astype(np.float64))
    g_lab = np.concatenate(labels)
    assert (g_lab == lab64).all()
    assert np.array_equal(counts.cpu().numpy(), np.bincount(lab64, minlength=k))
    assert len(empty) == ne64 == (1 if far else 0)
    if far:
        assert empty == [k // 2]
    # finalize leaves an empty cluster's centroid as it was; the oracle reseeds it
    keep = np.ones(k, bool)
    keep[empty] = False
    g_C = C_new.cpu().numpy()
    assert centroid_rel_err(C64[keep], g_C[keep]) < CENTROID_TOL[dt]
    assert np.array_equal(g_C[~keep], C0[~keep])
    if not far:
        assert rel_close(shift, shift64, 1e-6)
    obj = restated.objective(X.astype(np.float64), C0.astype(np.float64), lab64)
    assert rel_close(sq, obj, 1e-4 if dt == np.float32 else 1e-10)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("far", [False, True])
def test_train_spmd_one_rank_nccl(far):
    X, C0 = _blobs(30000, 160, 48, np.float64, seed=77, far_centroid=far)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        ops = DeviceShardOps(torch.from_numpy(X).cuda(), _native.KMB_FORM_PLAIN)
        C, lab, it, obj = train_spmd(ops, torch.from_numpy(C0).cuda(), 25, 0.0)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    Cr, labr, objr, itr = restated.train(X, C0, 25, 0.0)
    assert it == itr
    assert (lab.cpu().numpy() == labr).all()
    assert centroid_rel_err(Cr, C.cpu().numpy()) < 1e-12
    assert rel_close(obj, objr, 1e-10)


# ---- the library's own sharded loop (kmb_train_spmd) with torch.distributed callbacks ----

@pytest.mark.parametrize("far", [False, True])
def test_native_spmd_one_rank_equals_python_driver(far):
    """kmb_train_spmd over a one-rank NCCL group gives the Python driver's result
    bit for bit (same kernels, same exchange) and the FP64 oracle's training run."""
    from onedal_b200.spmd import train_spmd_native
    X, C0 = _blobs(30000, 160, 48, np.float64, seed=78, far_centroid=far)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
    try:
        Xd, Cd = torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()
        Cp, labp, itp, objp = train_spmd(DeviceShardOps(Xd, _native.KMB_FORM_PLAIN), Cd, 25, 0.0)
        Cn, labn, itn, objn = train_spmd_native(Xd, Cd, 25, 0.0)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert itn == itp
    assert np.array_equal(labn.cpu().numpy(), labp.cpu().numpy())
    assert np.array_equal(Cn.cpu().numpy(), Cp.cpu().numpy())
    assert rel_close(objn, objp, 1e-12)
    Cr, labr, objr, itr = restated.train(X, C0, 25, 0.0)
    assert itn == itr
    assert (labn.cpu().numpy() == labr).all()
    assert centroid_rel_err(Cr, Cn.cpu().numpy()) < 1e-12


def _native_rank(rank, world, port, X, C0, dt, q):
    import os
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch
    import torch.distributed as dist
    from onedal_b200.spmd import train_spmd_native
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        cut = np.linspace(0, X.shape[0], world + 1).astype(int)
        C, lab, it, obj = train_spmd_native(torch.from_numpy(X[cut[rank]:cut[rank + 1]]).cuda(),
                                            torch.from_numpy(C0).cuda(), 30, 0.0)
        torch.cuda.synchronize()
        q.put((rank, C.cpu().numpy(), lab.cpu().numpy(), it, obj))
    except Exception as e:  # reported to the parent
        q.put((rank, repr(e), None, None, None))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dt,far", [(np.float64, True), (np.float32, False), (np.float32, True)])
def test_native_spmd_two_ranks_gloo(dt, far):
    """Two ranks (two processes sharing the one GPU, gloo on the host as the
    communicator): identical centroids on both ranks, equal to the FP64 oracle's
    single-process run (responses, iterations, centroids), an emptied cluster
    reseeded across the ranks included. Float rows exchange the exact fixed-point
    sums, so their result is bit for bit the one-GPU train's (plain form)."""
    import torch.multiprocessing as mp
    from onedal_b200 import kmeans
    X, C0 = _blobs(24000, 40, 12, dt, seed=79, far_centroid=far)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_native_rank, args=(r, 2, port, X, C0, dt, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(2)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
    for r in res:
        assert r[2] is not None, r[1]
    (_, C0r, lab0, it0, obj0), (_, C1r, lab1, it1, obj1) = res
    assert it0 == it1 and np.array_equal(C0r, C1r) and obj0 == obj1
    Cr, labr, objr, itr = restated.train(X.astype(np.float64), C0.astype(np.float64), 30, 0.0)
    assert it0 == itr
    assert (np.concatenate([lab0, lab1]) == labr).all()
    assert centroid_rel_err(Cr, C0r) < CENTROID_TOL[dt]
    assert rel_close(obj0, objr, 1e-10 if dt == np.float64 else 1e-5)
    if dt == np.float32:
        desc = kmeans.descriptor(np.float32).set_cluster_count(C0.shape[0]).set_max_iteration_count(30) \
            .set_accuracy_threshold(0.0).set_compute_form(kmeans.compute_form.plain)
        one = kmeans.train(desc, X, C0)
        assert one.get_iteration_count() == it0
        assert np.array_equal(one.get_model().get_centroids(), C0r)
        assert np.array_equal(one.get_responses().ravel(), np.concatenate([lab0, lab1]))


def test_native_spmd_communicator_failure_is_reported():
    """A communicator callback that fails ends kmb_train_spmd with KMB_ECOMM (no
    hang, no device fault) and the context trains normally afterwards."""
    import ctypes
    X, C0 = _blobs(5000, 16, 6, np.float32, seed=80)
    Xd, Cd = torch.from_numpy(X).cuda(), torch.from_numpy(C0).cuda()
    ctx = _native.context(0)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    calls = {"allreduce": 0}

    def allgather(_user, send, nbytes, recv):
        ctypes.memmove(recv, send, nbytes)  # one rank
        return 0

    def allreduce_fails(_user, buf, count):
        calls["allreduce"] += 1
        return 1

    ar, ag = _native.ALLREDUCE_F64_FN(allreduce_fails), _native.ALLGATHER_FN(allgather)
    comm = _native.kmb_communicator(None, 0, 1, ar, ag)
    C = torch.empty_like(Cd)
    lab = torch.empty(X.shape[0], dtype=torch.int32, device="cuda")
    p = _native.kmb_params(6, 10, 0.0, _native.KMB_FORM_PLAIN, 0)
    obj, it = ctypes.c_double(), ctypes.c_int64()
    rc = ctx.lib.kmb_train_spmd(ctx.handle, _native.KMB_F32, Xd.data_ptr(), X.shape[0], X.shape[1], Cd.data_ptr(),
                                ctypes.byref(p), ctypes.byref(comm), C.data_ptr(), lab.data_ptr(), ctypes.byref(obj),
                                ctypes.byref(it))
    assert rc == _native.KMB_ECOMM and calls["allreduce"] == 1
    # the same context, a working one-rank communicator: the one-GPU train's result
    ok = _native.ALLREDUCE_F64_FN(lambda _u, _b, _c: 0)
    comm = _native.kmb_communicator(None, 0, 1, ok, ag)
    ctx.check(ctx.lib.kmb_train_spmd(ctx.handle, _native.KMB_F32, Xd.data_ptr(), X.shape[0], X.shape[1],
                                     Cd.data_ptr(), ctypes.byref(p), ctypes.byref(comm), C.data_ptr(), lab.data_ptr(),
                                     ctypes.byref(obj), ctypes.byref(it)))
    from onedal_b200 import kmeans
    desc = kmeans.descriptor(np.float32).set_cluster_count(6).set_max_iteration_count(10) \
        .set_compute_form(kmeans.compute_form.plain)
    one = kmeans.train(desc, X, C0)
    assert it.value == one.get_iteration_count()
    assert np.array_equal(C.cpu().numpy(), one.get_model().get_centroids())
