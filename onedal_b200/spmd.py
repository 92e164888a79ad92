"""Row-sharded (SPMD) k-means Lloyd training: one process per GPU.

Each rank holds a contiguous block of rows. Per iteration:

1. local statistics under the shared centroids C (``kmb_partial_sums``):
   labels, FP64 per-cluster sums, int64 counts, squared distances per row;
2. one all-reduce of a packed FP64 buffer [sums (k*d) | counts (k) | sum of
   squared distances (1)] (NCCL on GPUs; gloo in the CPU tests of this
   module's host logic); counts travel as doubles, exact below 2^53;
3. identical finalize on every rank (``kmb_finalize_centroids``):
   c_j = F(S_j / count_j), shift over non-empty clusters, list of empty ones;
4. when clusters are empty: every rank proposes its local top-m rows by squared
   distance, the proposals are all-gathered, and the global top-m by (distance
   descending, global row ascending) reseed the empty clusters in ascending
   cluster order -- DAAL's order (cpp/daal/src/algorithms/kmeans/
   kmeans_lloyd_batch_impl.i:153-188, kmeans_lloyd_impl.i:413-480);
5. stop when the shift <= eps, as kmeans_lloyd_batch_impl.i:189-212.

This mirrors the reference's SPMD exchange
(cpp/oneapi/dal/algo/kmeans/backend/gpu/cluster_updater.hpp:117-153,
backend/gpu/empty_cluster_handling_dpc.cpp:273-300) with FP64 sums instead of
per-rank F centroids, so every rank ends with bit-identical centroids.

The per-rank compute is a ``ShardOps`` object; ``DeviceShardOps`` calls the
CUDA library. The CPU tests supply a numpy implementation of the same two
methods to exercise the exchange logic with gloo ranks.
"""
import ctypes
from dataclasses import dataclass

import numpy as np
import torch
import torch.distributed as dist

from . import _native


@dataclass
class ShardStats:
    labels: torch.Tensor      # (n_local,) int32
    sums: torch.Tensor        # (k, d) float64
    counts: torch.Tensor      # (k,) int64
    row_sq: torch.Tensor      # (n_local,) squared distance of each row to its centroid
    sq_total: object          # this shard's sum of squared distances (a device tensor or a float)


class DeviceShardOps:
    """Per-rank compute on this process's GPU through the C ABI."""

    def __init__(self, X: torch.Tensor, form: int = _native.KMB_FORM_PLAIN):
        assert X.is_cuda and X.dim() == 2
        self.X = X.contiguous()
        self.form = form
        self.ctx = _native.context(X.device.index or 0)
        self.dtype = _native.KMB_F32 if X.dtype == torch.float32 else _native.KMB_F64

    def partial(self, C: torch.Tensor) -> ShardStats:
        n, d = self.X.shape
        k = C.shape[0]
        dev = self.X.device
        labels = torch.empty(n, dtype=torch.int32, device=dev)
        sums = torch.empty((k, d), dtype=torch.float64, device=dev)
        counts = torch.empty(k, dtype=torch.int64, device=dev)
        sq = torch.zeros(1, dtype=torch.float64, device=dev)
        row_sq = torch.empty(n, dtype=self.X.dtype, device=dev)
        self.ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        self.ctx.check(self.ctx.lib.kmb_partial_sums(self.ctx.handle, self.dtype, self.X.data_ptr(), n, d,
                                                     C.data_ptr(), k, self.form, labels.data_ptr(), sums.data_ptr(),
                                                     counts.data_ptr(), sq.data_ptr(), row_sq.data_ptr()))
        return ShardStats(labels, sums, counts, row_sq, sq)  # sq stays on the device: no sync here

    def finalize(self, sums: torch.Tensor, counts: torch.Tensor, C: torch.Tensor):
        k, d = C.shape
        C_new = torch.empty_like(C)
        empty = torch.empty(k, dtype=torch.int32, device=C.device)
        shift = ctypes.c_double()
        ne = ctypes.c_int64()
        self.ctx.check(self.ctx.lib.kmb_finalize_centroids(self.ctx.handle, self.dtype, sums.data_ptr(),
                                                           counts.data_ptr(), C.data_ptr(), k, d, C_new.data_ptr(),
                                                           ctypes.byref(shift), empty.data_ptr(), ctypes.byref(ne)))
        return C_new, shift.value, empty[: ne.value].cpu().tolist()

    def rows(self, local_idx):
        return self.X[local_idx.to(device=self.X.device, dtype=torch.long)]


def _top_candidates(row_sq: torch.Tensor, m: int, row_offset: int):
    """This rank's m largest squared distances in (value descending, global row
    ascending) order, computed where row_sq lives: the distances are not copied to
    the host. NaN distances order last (as -inf)."""
    n = row_sq.shape[0]
    take = min(m, n)
    v = torch.nan_to_num(row_sq.to(torch.float64), nan=float("-inf"))
    # a stable descending sort keeps equal values in ascending row order
    order = torch.sort(v, descending=True, stable=True).indices[:take]
    vals = torch.full((m,), float("-inf"), dtype=torch.float64, device=row_sq.device)
    rows = torch.full((m,), np.iinfo(np.int64).max, dtype=torch.int64, device=row_sq.device)
    vals[:take] = v[order]
    rows[:take] = order + row_offset
    return vals, rows, order


def exchange(st: ShardStats, group=None):
    """The iteration's one collective: all-reduce of [sums | counts | squared
    distances] packed into one FP64 buffer. Returns (sums, counts, sq_total) summed
    over the ranks, on the sums' device."""
    k, d = st.sums.shape
    dev = st.sums.device
    packed = torch.empty(k * d + k + 1, dtype=torch.float64, device=dev)
    packed[: k * d] = st.sums.reshape(-1)
    packed[k * d: k * d + k] = st.counts.to(torch.float64)
    packed[k * d + k:] = torch.as_tensor(st.sq_total, dtype=torch.float64, device=dev).reshape(1)
    dist.all_reduce(packed, group=group)
    return (packed[: k * d].view(k, d), packed[k * d: k * d + k].round().to(torch.int64),
            packed[k * d + k:])


def train_spmd(ops, C0: torch.Tensor, max_iteration_count: int, accuracy_threshold: float = 0.0, group=None):
    """Runs the sharded Lloyd loop. Returns (centroids, local labels, iterations, objective)
    with centroids identical on every rank."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    dev = C0.device
    n_local = torch.tensor([ops.X.shape[0]], dtype=torch.int64, device=dev)
    sizes = [torch.zeros_like(n_local) for _ in range(world)]
    dist.all_gather(sizes, n_local, group=group)
    offsets = np.cumsum([0] + [int(s.item()) for s in sizes])
    row_offset = int(offsets[rank])

    C = C0.clone()
    it = 0
    while it < max_iteration_count:
        st = ops.partial(C)
        sums, counts, _ = exchange(st, group)
        C_new, shift, empty = ops.finalize(sums, counts, C)
        m = len(empty)
        if m:
            vals, rows, local = _top_candidates(st.row_sq, m, row_offset)
            d = C.shape[1]
            payload_rows = torch.zeros((m, d), dtype=C.dtype, device=dev)
            if len(local):
                payload_rows[: len(local)] = ops.rows(local).to(C.dtype)
            v_t = vals.to(dev)
            r_t = rows.to(dev)
            gv = [torch.empty_like(v_t) for _ in range(world)]
            gr = [torch.empty_like(r_t) for _ in range(world)]
            gx = [torch.empty_like(payload_rows) for _ in range(world)]
            dist.all_gather(gv, v_t, group=group)
            dist.all_gather(gr, r_t, group=group)
            dist.all_gather(gx, payload_rows, group=group)
            av = torch.cat(gv).cpu().numpy()
            ar = torch.cat(gr).cpu().numpy()
            ax = torch.cat(gx)
            order = np.lexsort((ar, -av))[:m]
            if not np.isfinite(av[order]).all():
                raise RuntimeError("number of clusters exceeds the number of points")
            for e, cid in enumerate(empty):
                row = ax[int(order[e])]
                shift += float(((C[cid].double() - row.double()) ** 2).sum())
                C_new[cid] = row
        C = C_new
        it += 1
        if shift <= accuracy_threshold:
            break
    # responses and objective under the final centroids
    st = ops.partial(C)
    obj = torch.as_tensor(st.sq_total, dtype=torch.float64, device=dev).reshape(1).clone()
    dist.all_reduce(obj, group=group)
    return C, st.labels, it, float(obj.item())


def train_spmd_native(X: torch.Tensor, C0: torch.Tensor, max_iteration_count: int, accuracy_threshold: float = 0.0,
                      form: int = _native.KMB_FORM_PLAIN, group=None):
    """The same sharded Lloyd loop run by the library itself (kmb_train_spmd), with
    torch.distributed as its communicator: one host allreduce of the packed FP64
    [sums | counts | squared distances] per iteration and one allgather of the reseed
    candidates when clusters are empty. X is this rank's block of rows (CUDA), C0 the
    common initial centroids. Returns (centroids, local labels, iterations, objective);
    the centroids are identical on every rank. With NCCL the host buffers go through
    device copies; with gloo they are reduced in place."""
    assert X.is_cuda and C0.is_cuda and X.dim() == 2
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nccl = dist.get_backend(group) == "nccl"
    dev = X.device
    X = X.contiguous()
    C0 = C0.contiguous().to(X.dtype)

    def allreduce(_user, buf, count):
        try:
            host = torch.from_numpy(np.ctypeslib.as_array(buf, shape=(count,)))  # the library's buffer, in place
            if nccl:
                t = host.to(dev)
                dist.all_reduce(t, group=group)
                host.copy_(t.cpu())
            else:
                dist.all_reduce(host, group=group)
            return 0
        except Exception:  # reported to the library as a communicator failure
            return 1

    def allgather(_user, send, nbytes, recv):
        try:
            src = torch.from_numpy(np.ctypeslib.as_array((ctypes.c_uint8 * nbytes).from_address(send))).clone()
            dst = torch.from_numpy(np.ctypeslib.as_array((ctypes.c_uint8 * (nbytes * world)).from_address(recv)))
            if nccl:
                outs = [torch.empty(nbytes, dtype=torch.uint8, device=dev) for _ in range(world)]
                dist.all_gather(outs, src.to(dev), group=group)
            else:
                outs = [torch.empty(nbytes, dtype=torch.uint8) for _ in range(world)]
                dist.all_gather(outs, src, group=group)
            dst.copy_(torch.cat(outs).cpu())
            return 0
        except Exception:
            return 1

    ar_cb = _native.ALLREDUCE_F64_FN(allreduce)
    ag_cb = _native.ALLGATHER_FN(allgather)
    comm = _native.kmb_communicator(None, rank, world, ar_cb, ag_cb)
    n, d = X.shape
    k = C0.shape[0]
    ctx = _native.context(dev.index or 0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    C = torch.empty_like(C0)
    labels = torch.empty(n, dtype=torch.int32, device=dev)
    params = _native.kmb_params(k, int(max_iteration_count), float(accuracy_threshold), int(form), 0)
    obj = ctypes.c_double()
    it = ctypes.c_int64()
    dtype = _native.KMB_F32 if X.dtype == torch.float32 else _native.KMB_F64
    ctx.check(ctx.lib.kmb_train_spmd(ctx.handle, dtype, X.data_ptr(), n, d, C0.data_ptr(), ctypes.byref(params),
                                     ctypes.byref(comm), C.data_ptr(), labels.data_ptr(), ctypes.byref(obj),
                                     ctypes.byref(it)))
    return C, labels, it.value, obj.value
