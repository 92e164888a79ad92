"""Benchmark: k-means Lloyd iterations/s on the precision workload
(n=20,000,000, d=128, k=1024, float32 input), one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form bf16|bf16x3|plain] [--impl b200|reference]

A step is one Lloyd iteration (assignment + centroid update) over all rows,
inputs resident in HBM (10.24 GB of rows, far larger than the 126 MB L2, so no
L2 flush is needed between steps). `value` = whole-job iterations/s timed with
CUDA events on the launching stream between barriers, max over ranks. `e2e` is
the same metric through the public API (kmeans.train on pinned host buffers:
host->device copy of the rows, the K iterations, the final responses/objective
pass and the device->host copy of centroids and responses inside the timed
region). `roofline` is for the dominant kernel (the assignment), its per-launch
duration measured with CUDA events recorded by the library on its stream.
`cpu_baseline` is the reference's own DAAL kernel (oracle/_ref) on the host cores.

With --impl reference, rank 0 times the reference DAAL kernel on the host cores
(a bounded row sample of the same workload, scaled to the full row count) and
prints the same metric; other ranks exit.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
# (526.31 MB read + 10.91 MB written) / 1,000,000 rows, assign_tc_kernel at d=128, k=1024
TC_DRAM_BYTES_PER_ROW = 537.21
sys.path.insert(0, ROOT)

METRIC = "Lloyd iter/s n=20M,d=128,k=1024 BF16-TC vs FP32 plain; p50/p99 infer latency"
UNIT = "iter/s"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_iters_per_s(X_host, C0_host, n_full, iters, threads):
    """Reference DAAL kernel on the given rows: per-iteration time from a train with
    `iters` iterations minus an infer pass (the train's final responses+objective),
    scaled to n_full rows when the rows are a sample."""
    from oracle import daal_ref
    daal_ref.set_threads(threads)
    t0 = time.perf_counter()
    daal_ref.infer(X_host, C0_host, True)
    t_inf = time.perf_counter() - t0
    t0 = time.perf_counter()
    _, _, _, it = daal_ref.train(X_host, C0_host, iters, 0.0)
    t_tr = time.perf_counter() - t0
    per_iter = max(t_tr - t_inf, 1e-9) / max(it, 1)
    scale = n_full / X_host.shape[0]
    return 1.0 / (per_iter * scale), per_iter, it


def run_plusplus(args, X, ctx):
    """k-means++ initialisation (the default init of train() without initial centroids)
    over the resident rows: centers/s, with each round's pass over X against the HBM
    roofline, and the reference kernel's rounds on a row sample on the host cores."""
    import numpy as np
    import torch

    from onedal_b200 import kmeans
    n, d = X.shape
    k = args.plusplus_k
    stream = torch.cuda.current_stream()
    kmeans.init_plusplus(X, min(k, 8), np.float32, ctx=ctx)  # warm-up (allocations, module load)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    kmeans.init_plusplus(X, k, np.float32, ctx=ctx)
    e1.record(stream)
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / 1e3
    peaks, src = load_peaks()
    bytes_per_round = n * d * 4 + 2 * n * 4  # rows read, running minima read + written
    achieved = bytes_per_round * (k - 1) / s / 1e9
    out = {"metric": "k-means++ centers/s", "value": (k - 1) / s, "unit": "centers/s", "k": k, "seconds": s,
           "ms_per_center": s / (k - 1) * 1e3,
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": achieved / peaks["hbm_gbs"], "peak_source": src,
                        "algorithmic_bytes_per_round": bytes_per_round,
                        "note": "whole rounds (distance update + sampling walk) against the rows' bytes"}}
    if args.cpu_sample_rows > 0:
        from oracle import daal_ref
        if daal_ref.available():
            ns = min(args.cpu_sample_rows, n)
            kc = 64
            Xs = X[:ns].cpu().numpy()
            daal_ref.set_threads(os.cpu_count() or 1)
            t0 = time.perf_counter()
            daal_ref.init_plusplus(Xs, kc)
            per_round = (time.perf_counter() - t0) / (kc - 1) * (n / ns)
            out["cpu_baseline"] = {"value": 1.0 / per_round, "unit": "centers/s", "cores": os.cpu_count(),
                                   "kind": "reference",
                                   "sample": f"reference plusPlus init kernel, first {ns} of {n} rows, {kc} centers, "
                                             f"per-center time scaled by rows"}
    return out


def measured_fma_peak_tflops(device=0, dtype=0):
    """The device's FMA peak measured by the library's microbenchmark
    (kmb_measure_fma_peak), TFLOP/s: FP64 for dtype 1; for FP32 the larger of the
    scalar FMA and the packed pair FMA (fma.rn.f32x2) the plain kernel issues."""
    import ctypes

    from onedal_b200 import _native
    lib = _native.load_library()
    best = None
    for dt in ((0, 2) if dtype == 0 else (dtype,)):
        g = ctypes.c_double()
        if lib.kmb_measure_fma_peak(device, dt, ctypes.byref(g)) == 0:
            best = max(best or 0.0, g.value / 1e3)
    return best


def run_plain_scale(args, ctx, device=0):
    """Plain FP32 form at scale: n = 10,000,000 rows, d = 64, k = 256, float32, 256
    anisotropic blobs (per-blob diagonal std log-uniform in [0.3, 3], centres
    U[-20,20]^64, Dirichlet(1) weights), initial centroids a seeded row sample,
    exactly 20 Lloyd iterations (eps 0; the loop runs all 20 unless it reaches an
    exact fixed point), inputs resident in HBM (2.56 GB, above L2). Reports Lloyd
    iterations/s and the assignment kernel against the measured FP32 FMA peak."""
    import ctypes

    import torch

    from onedal_b200 import _native, workloads
    w = workloads.PLAIN_GPU
    X, C0 = workloads.make(w, "cuda", args.plain_scale_rows or w.n)
    n, d = X.shape
    k = C0.shape[0]
    labels = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def iterate(T, C):
        p = _native.kmb_params(k, T, 0.0, _native.KMB_FORM_PLAIN, 0)
        it = ctypes.c_int64()
        ctx.check(ctx.lib.kmb_lloyd_iterate(ctx.handle, _native.KMB_F32, X.data_ptr(), n, d, C.data_ptr(),
                                            ctypes.byref(p), labels.data_ptr(), ctypes.byref(it), None))
        return it.value

    iterate(3, C0.clone())
    torch.cuda.synchronize()
    C = C0.clone()
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 1))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    it = iterate(w.iterations, C)
    e1.record(stream)
    torch.cuda.synchronize()
    kt, kl = ctypes.c_double(), ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 0, ctypes.byref(kt), ctypes.byref(kl)))
    ut, ul = ctypes.c_double(), ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 2, ctypes.byref(ut), ctypes.byref(ul)))
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 0))
    s = e0.elapsed_time(e1) / 1e3
    kms = kt.value / max(kl.value, 1)
    flops = 2.0 * n * k * d
    achieved = flops / (kms / 1e3) / 1e12
    peak = measured_fma_peak_tflops(device, 0)
    out = {"metric": "Lloyd iter/s (plain FP32 form)", "value": it / s, "unit": "iter/s", "iterations": it,
           "ms_per_iteration": s / max(it, 1) * 1e3,
           "config": {"workload": f"plain at scale n={n} d={d} k={k} float32, {k} anisotropic blobs, "
                                  "Dirichlet(1) weights", "n": n, "d": d, "k": k,
                      "l2": f"inputs ({n * d * 4 / 1e9:.2f} GB) larger than L2; no flush"},
           "roofline": {"bound": "fp32_fma", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                        "frac": achieved / peak if peak else None,
                        "peak_source": "FP32 FMA peak measured on this GPU (kmb_measure_fma_peak, larger of scalar and packed-pair FMA)",
                        "kernel_ms_avg": kms, "kernel_launches": kl.value,
                        "update_ms_avg": ut.value / max(ul.value, 1),
                        "algorithmic_flops_per_launch": flops, "algorithmic_bytes_per_launch": 4 * n * d + 8 * n,
                        "traffic": None}}
    del X
    torch.cuda.empty_cache()
    return out


def run_csr(args, ctx):
    """method::lloyd_csr on a synthetic sparse workload held in HBM: n = 2M rows,
    d = 20,000 columns, 64 stored entries per row (uniform columns, one per
    312-column stripe, N(0, 1) values), k = 256 centroids started from k rows,
    float32, 10 iterations (eps 0). Reports Lloyd iterations/s of the whole train
    call (the final responses pass and objective included), the assignment
    kernel's FLOP rate and its centroid-gather bytes, and the CSR oracle port on a
    20,000-row sample on the host cores, scaled by rows."""
    import ctypes

    import numpy as np
    import torch

    from onedal_b200 import _native, kmeans
    n, d, per, k, T = args.csr_rows, 20000, 64, 256, 10
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    stripe = d // per
    cols = (torch.randint(0, stripe, (n, per), device="cuda", generator=g)
            + torch.arange(per, device="cuda") * stripe).to(torch.int64).reshape(-1)
    vals = torch.randn(n * per, device="cuda", generator=g, dtype=torch.float32)
    offs = torch.arange(0, n * per + 1, per, device="cuda", dtype=torch.int64)
    table = kmeans.csr_table(vals, cols, offs, n, d, kmeans.sparse_indexing.zero_based)
    pick = torch.randperm(n, device="cuda", generator=g)[:k]
    C0 = torch.zeros((k, d), device="cuda")
    rows_idx = (pick[:, None] * per + torch.arange(per, device="cuda")[None, :]).reshape(-1)
    C0[torch.arange(k, device="cuda").repeat_interleave(per), cols[rows_idx]] = vals[rows_idx]
    desc = kmeans.descriptor(np.float32, kmeans.method.lloyd_csr).set_cluster_count(k).set_max_iteration_count(T)
    kmeans.train(desc.set_max_iteration_count(1), table, C0)  # warm-up
    desc.set_max_iteration_count(T)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 1))
    e0.record(stream)
    r = kmeans.train(desc, table, C0)
    e1.record(stream)
    torch.cuda.synchronize()
    kt, kl = ctypes.c_double(), ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 0, ctypes.byref(kt), ctypes.byref(kl)))
    ut, ul = ctypes.c_double(), ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 2, ctypes.byref(ut), ctypes.byref(ul)))
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 0))
    s = e0.elapsed_time(e1) / 1e3
    it = r.get_iteration_count()
    assign_ms = kt.value / max(kl.value, 1)
    nnz = n * per
    out = {"metric": "CSR Lloyd iter/s", "value": it / s, "unit": "iter/s", "iterations": it, "seconds": s,
           "config": {"workload": f"synthetic CSR n={n} d={d} {per} stored entries per row, k={k}, float32",
                      "nnz": nnz},
           "assign_ms_avg": assign_ms, "update_ms_avg": ut.value / max(ul.value, 1),
           "assign_tflops": 2.0 * nnz * k / (assign_ms / 1e3) / 1e12,
           "assign_centroid_gather_gbs": nnz * k * 4 / (assign_ms / 1e3) / 1e9}
    if args.cpu_sample_rows > 0:
        from oracle import restated
        ns = 20000
        v = vals[:ns * per].cpu().numpy()
        c = cols[:ns * per].cpu().numpy()
        o = offs[:ns + 1].cpu().numpy()
        t0 = time.perf_counter()
        _, _, _, itc = restated.train_csr(v, c, o, d, C0.cpu().numpy(), 2, 0.0)
        per_iter = (time.perf_counter() - t0) / 3 * (n / ns)  # 2 updates + the final pass
        out["cpu_baseline"] = {"value": 1.0 / per_iter, "unit": "iter/s", "cores": os.cpu_count(), "kind": "port",
                               "sample": f"CSR oracle (OpenMP) on the first {ns} of {n} rows, 2 iterations + final "
                                         f"pass, per-pass time scaled by rows"}
    return out


def make_workload(device, n=None):
    import torch
    from onedal_b200 import workloads
    X, C0 = workloads.make(workloads.PRECISION, device, n=n)
    torch.cuda.synchronize()
    return X, C0


def reference_rows(w):
    """The workload's rows and initial centroids on the host, drawn by the same
    generator as the GPU arm's (on the GPU when one is present, so both arms see
    identical data; the reference itself never touches the GPU)."""
    import torch
    from onedal_b200 import workloads
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    X, C0 = workloads.make(w, dev)
    Xh = X.cpu().numpy()
    Ch = C0.cpu().numpy()
    del X, C0
    if dev == "cuda":
        torch.cuda.empty_cache()
    return Xh, Ch, dev


def run_reference(args):
    """The reference's own DAAL Lloyd kernel (oracle/_ref, built from the reference
    sources) on all host cores, at the full configuration: n = 20,000,000 rows, d =
    128, k = 1024, float32. Warm-up: one train call of `warmup` iterations. Timed: one
    train call of `steps` iterations minus the final responses + objective pass it
    ends with (timed separately as an infer call on the same rows), so ms_per_step
    is one Lloyd iteration over all 20M rows."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from onedal_b200 import workloads
    from oracle import daal_ref
    w = workloads.PRECISION
    if not daal_ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference kernel library oracle/_ref not built"}))
        return
    Xh, Ch, gen = reference_rows(w)
    n = Xh.shape[0]
    threads = os.cpu_count() or 1
    daal_ref.set_threads(threads)
    if args.warmup > 0:
        daal_ref.train(Xh, Ch, args.warmup, 0.0)
    t0 = time.perf_counter()
    C, _, _, it = daal_ref.train(Xh, Ch, args.steps, 0.0)
    t_train = time.perf_counter() - t0
    t0 = time.perf_counter()
    daal_ref.infer(Xh, C, True)
    t_final = time.perf_counter() - t0
    per_iter = max(t_train - t_final, 1e-9) / max(it, 1)
    v = 1.0 / per_iter
    sample = (f"all {n} rows, {it} Lloyd iterations of one train call minus its final responses+objective "
              f"pass (timed as an infer call), {threads} threads, OpenBLAS sgemm")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_iter * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(n, w.d, w.k),
        "impl": "reference",
        "reference_kernel": "DAAL KMeansBatchKernel<lloydDense, float> built from the reference sources",
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timing": {"train_s": t_train, "final_pass_s": t_final, "iterations": it, "rows_generated_on": gen},
    }
    print(json.dumps(line))


def workload_config(n, d, k):
    """The `config` object both arms report for the precision workload."""
    return {"workload": f"precision n={n} d={d} k={k} float32, {k} blobs std 1 in U[-5,5]^{d}, "
                        "10% bisector near-ties", "n": n, "d": d, "k": k,
            "l2": f"inputs ({n * d * 4 / 1e9:.2f} GB) larger than L2; no flush"}


def run_serving(args, device=0):
    """Serving form: 64 resident centroid sets, a Poisson stream of infer (90%) and small
    train (10%) requests; saturation throughput, then p50/p99 latency at fractions of it."""
    import threading

    import numpy as np
    import torch

    from onedal_b200 import _native
    from onedal_b200.serving import KMeansServer

    rng = np.random.default_rng(1005)
    n_models = 64
    ks = np.exp(rng.uniform(np.log(16), np.log(4096), n_models)).astype(int)
    ds = rng.choice([32, 64, 128, 256], n_models)
    models = [rng.uniform(-1, 1, (int(k), int(d))).astype(np.float32) for k, d in zip(ks, ds)]
    pool_rows = 1 << 20
    pools = {}
    for dd in (32, 64, 128, 256):  # pinned N(0,1) rows per width; request rows are contiguous slices
        t = torch.empty((pool_rows, dd), dtype=torch.float32, pin_memory=True)
        t.normal_(generator=torch.Generator().manual_seed(dd))
        pools[dd] = (t, t.numpy())
    # small-train datasets (Gaussian mixtures), reused by the train requests
    trains = []
    for i in range(8):
        k = int(rng.integers(2, 65))
        d = int(rng.choice([32, 64, 128, 256]))
        n = int(rng.integers(max(k, 5000), 50_001))
        c = rng.uniform(-10, 10, (k, d))
        X = (c[rng.integers(0, k, n)] + rng.standard_normal((n, d))).astype(np.float32)
        trains.append((X, X[:k].copy()))

    def make_requests(count, seed):
        g = np.random.default_rng(seed)
        out = []
        for _ in range(count):
            if g.random() < 0.9:
                m = int(g.integers(0, n_models))
                n = int(min(1_000_000, max(1, round(g.lognormal(np.log(4096), 1.5)))))
                d = models[m].shape[1]
                off = int(g.integers(0, pool_rows - n + 1))
                out.append(("infer", m, pools[d][1][off:off + n]))
            else:
                out.append(("train", int(g.integers(0, len(trains))), None))
        return out

    def submit(srv, ids, req):
        kind, m, X = req
        if kind == "infer":
            return srv.submit_infer(ids[m], X)
        Xt, C0 = trains[m]
        return srv.submit_train(Xt, C0, 15)

    def run_point(srv, ids, reqs, rate):
        """rate=None: everything at t=0 (saturation); else Poisson arrivals at `rate` per s."""
        g = np.random.default_rng(77)
        handles = [None] * len(reqs)
        lat = {}
        queued = {}
        done = threading.Event()

        def collector():
            for i in range(len(reqs)):
                while handles[i] is None:
                    time.sleep(0.0001)
                _, (l, qd) = srv.wait(handles[i], timeout=600, detail=True)
                lat[i] = l
                queued[i] = qd
            done.set()

        prepared = reqs
        th = threading.Thread(target=collector)
        th.start()
        t0 = time.perf_counter()
        t_next = t0
        for i, req in enumerate(prepared):
            if rate:
                t_next += g.exponential(1.0 / rate)
                while time.perf_counter() < t_next:
                    pass
            handles[i] = submit(srv, ids, req)
        done.wait()
        t1 = time.perf_counter()
        th.join()
        inf = [lat[i] for i, r in enumerate(reqs) if r[0] == "infer"]
        tc_form = _native.KMB_FORM_BF16X3
        forms = [srv.infer_form(ids[r[1]], r[2].shape[0]) if r[0] == "infer" else None for r in reqs]
        by = {f: [lat[i] for i, r in enumerate(reqs) if r[0] == "infer" and forms[i] == f]
              for f in (_native.KMB_FORM_PLAIN, tc_form)}
        byq = {f: [queued[i] for i, r in enumerate(reqs) if r[0] == "infer" and forms[i] == f]
               for f in (_native.KMB_FORM_PLAIN, tc_form)}
        cls = {name: {"requests": len(by[f]), "p50_ms": float(np.percentile(by[f], 50) * 1e3) if by[f] else None,
                      "p99_ms": float(np.percentile(by[f], 99) * 1e3) if by[f] else None,
                      "queued_p50_ms": float(np.percentile(byq[f], 50) * 1e3) if byq[f] else None,
                      "queued_p99_ms": float(np.percentile(byq[f], 99) * 1e3) if byq[f] else None}
               for name, f in (("grouped_plain", _native.KMB_FORM_PLAIN), ("tensor_core", tc_form))}
        return {"requests": len(reqs), "seconds": t1 - t0, "throughput_rps": len(reqs) / (t1 - t0),
                "p50_ms": float(np.percentile(inf, 50) * 1e3), "p99_ms": float(np.percentile(inf, 99) * 1e3),
                "by_form": cls,
                "train_p50_ms": float(np.percentile([lat[i] for i, r in enumerate(reqs) if r[0] == "train"] or [0],
                                                    50) * 1e3)}

    def unloaded(srv, ids, reqs):
        """Each infer request alone on the idle server (submit, wait, next): the latency
        floor of the request mix, with no queueing and no sharing of the device."""
        lat = []
        for kind, m, X in reqs:
            if kind == "infer":
                lat.append(srv.wait(srv.submit_infer(ids[m], X), timeout=600)[1])
        return {"requests": len(lat), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3)}

    with KMeansServer(device=device, hbm_budget_bytes=60 << 30, lanes=args.serving_lanes, trainers=6) as srv:
        ids = [srv.add_model(C) for C in models]
        run_point(srv, ids, make_requests(200, 1), None)  # warm-up
        floor = unloaded(srv, ids, make_requests(max(args.serving_requests // 10, 200), 9))
        sat = run_point(srv, ids, make_requests(args.serving_requests, 2), None)
        points = []
        for frac in (0.5, 0.8):
            rate = frac * sat["throughput_rps"]
            pt = run_point(srv, ids, make_requests(args.serving_requests, 3 + int(frac * 10)), rate)
            pt["offered_rps"] = rate
            pt["fraction_of_saturation"] = frac
            points.append(pt)
        st = srv.stats()
    return {"saturation_rps": sat["throughput_rps"], "saturation_p99_ms": sat["p99_ms"], "unloaded": floor,
            "points": points,
            "models": n_models, "budget_bytes": 60 << 30, "lanes": args.serving_lanes, "trainers": 6,
            "mean_requests_per_batch": st["batched_requests"] / max(st["batches"], 1),
            "peak_in_use_bytes": st["peak_in_use_bytes"],
            "note": "p50/p99 = host submit->completion of infer requests; rows from a pinned pool"}


def run_sharded(args, dist, world, rank, local, form):
    """N > 1: weak scaling. Each rank holds its own 20M-row shard of an N x 20M-row
    problem (same generator, seed + rank) and the ranks run Lloyd iterations with one
    FP64 all-reduce of [sums | counts] per iteration (onedal_b200.spmd). value =
    shards x iterations / s (iterations/s of 20M-row shards processed by the job)."""
    import torch

    from onedal_b200 import spmd, workloads

    w = workloads.PRECISION
    n = args.rows or w.n
    X, _ = workloads.make(workloads.Workload(w.name, n, w.d, w.k, w.iterations, w.eps, w.seed + rank), "cuda", n=n)
    C0 = workloads.make(w, "cpu", n=max(w.k, 100_000))[1].cuda()  # same initial centroids on every rank
    ops = spmd.DeviceShardOps(X, form)

    def iterate(C, T):
        for _ in range(T):
            st = ops.partial(C)
            sums, counts, _ = spmd.exchange(st)
            C, shift, empty = ops.finalize(sums, counts, C)
        return C

    iterate(C0.clone(), args.warmup)
    torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    iterate(C0.clone(), args.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = torch.tensor([e0.elapsed_time(e1)], device="cuda")
    dist.all_reduce(ms, op=dist.ReduceOp.MAX)
    ms = float(ms.item())
    if rank == 0:
        line = {
            "metric": METRIC, "value": world * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"precision, {n} rows per rank (seed + rank), d={w.d}, k={w.k}, float32",
                       "n_per_rank": n, "d": w.d, "k": w.k, "form": args.form,
                       "exchange": "one NCCL all-reduce per iteration of a packed FP64 buffer [sums (k*d) | counts (k) | squared distances (1)]",
                       "value_unit": "20M-row shard iterations per second, summed over ranks"},
        }
        print(json.dumps(line))
    dist.destroy_process_group()


def run_batched(args):
    """Batched form: `args.batched_problems` independent problems (n log-uniform in
    [1e3, 2e5], d in {8,16,32,64}, k log-uniform int in [4,128], Gaussian mixtures of
    k blobs, std 1, centres U[-10,10]^d), up to 30 iterations each, stop at shift 0,
    trained by one persistent kernel. Algorithmic work per problem iteration: 2nkd
    flops, and 8nd bytes (the rows read by the assignment and by the accumulation)."""
    import numpy as np
    import torch

    from onedal_b200.batched import batched_train

    g = np.random.default_rng(1004)
    tg = torch.Generator(device="cuda")
    tg.manual_seed(1004)
    probs = []
    for _ in range(args.batched_problems):
        n = int(np.exp(g.uniform(np.log(1e3), np.log(2e5))))
        d = int(g.choice([8, 16, 32, 64]))
        k = int(round(np.exp(g.uniform(np.log(4), np.log(128)))))
        centres = (torch.rand(k, d, generator=tg, device="cuda") * 20 - 10)
        lab = torch.randint(0, k, (n,), generator=tg, device="cuda")
        X = centres[lab] + torch.randn(n, d, generator=tg, device="cuda")
        C0 = X[torch.randperm(n, generator=tg, device="cuda")[:k]].clone()
        probs.append((X, C0))
    T = 30
    # autotune every (d, cluster tile) class present, then warm up (arena in the library's
    # memory pool), outside the timed call
    classes = {}
    for X, C0 in probs:
        kp = 16
        while kp < C0.shape[0]:
            kp *= 2
        classes.setdefault(((X.shape[1] + 7) // 8, kp), (X, C0))
    batched_train(list(classes.values()), 2)
    batched_train(probs, 1)  # warm: the library's pool then holds this call's arena
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    res, info = batched_train(probs, T, use_graph=True)
    e1.record()
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / 1e3
    ks = info["kernel_ms"] / 1e3 if info.get("kernel_ms", -1) > 0 else None
    fma_peak = measured_fma_peak_tflops(0, 0)
    hbm_peak = load_peaks()[0].get("hbm_gbs")
    iters = sum(r[2] for r in res)
    flops = sum(2.0 * X.shape[0] * C0.shape[0] * X.shape[1] * r[2] for (X, C0), r in zip(probs, res))
    nbytes = sum(8.0 * X.shape[0] * X.shape[1] * r[2] for (X, C0), r in zip(probs, res))
    return {"problems": len(probs), "iterations_each_max": T, "total_problem_iterations": iters,
            "seconds": s, "problem_iterations_per_s": iters / s, "rows": sum(p[0].shape[0] for p in probs),
            "row_iterations_per_s": sum(p[0].shape[0] * r[2] for p, r in zip(probs, res)) / s,
            "algorithmic_tflops": flops / s / 1e12, "algorithmic_gbs": nbytes / s / 1e9,
            "kernel_seconds": ks, "kernel_problem_iterations_per_s": iters / ks if ks else None,
            "roofline": {"bound": "latency (neither FFMA nor HBM)", "fma_peak_tflops": fma_peak,
                         "achieved_tflops": flops / ks / 1e12 if ks else None,
                         "fma_frac": (flops / ks / 1e12) / fma_peak if ks and fma_peak else None,
                         "achieved_gbs": nbytes / ks / 1e9 if ks else None,
                         "hbm_peak_gbs": hbm_peak, "hbm_frac": (nbytes / ks / 1e9) / hbm_peak if ks and hbm_peak else None,
                         "note": "the persistent kernel alone (CUDA events in the library, kmb_batched_info.kernel_ms) "
                                 "against the FP32 FMA and HBM peaks"},
            "variants": info["variants"], "classes": len(classes),
            "note": "seconds: one whole call (arena, work lists, autotuned tiles, then row norms, scales and every "
                    "iteration in one kernel); kernel_seconds: that kernel alone"}


def run_b200(args):
    import ctypes

    import numpy as np
    import torch

    from onedal_b200 import _native, kmeans, workloads

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    w = workloads.PRECISION
    form = {"bf16x3": _native.KMB_FORM_BF16X3, "bf16": _native.KMB_FORM_BF16}.get(args.form, _native.KMB_FORM_PLAIN)
    tc_form = form != _native.KMB_FORM_PLAIN
    if world > 1:
        return run_sharded(args, dist, world, rank, local, form)

    X, C0 = make_workload("cuda", n=args.rows)
    n, d = X.shape
    k = C0.shape[0]
    ctx = _native.context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    labels = torch.empty(n, dtype=torch.int32, device="cuda")
    C = C0.clone()

    def iterate(T, Cbuf):
        p = _native.kmb_params(k, T, 0.0, form, 0)
        it = ctypes.c_int64()
        st = _native.kmb_stats()
        ctx.check(ctx.lib.kmb_lloyd_iterate(ctx.handle, _native.KMB_F32, X.data_ptr(), n, d, Cbuf.data_ptr(),
                                            ctypes.byref(p), labels.data_ptr(), ctypes.byref(it), ctypes.byref(st)))
        return it.value, st

    # warm-up
    iterate(args.warmup, C)
    torch.cuda.synchronize()
    C.copy_(C0)

    sampler = ClockSampler(local)
    sampler.start()
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 1))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    iters_done, st = iterate(args.steps, C)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    kernel_id = 1 if tc_form else 0
    kt = ctypes.c_double()
    kl = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, kernel_id, ctypes.byref(kt), ctypes.byref(kl)))
    ut = ctypes.c_double()
    ul = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 2, ctypes.byref(ut), ctypes.byref(ul)))
    rt = ctypes.c_double()
    rl = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 4, ctypes.byref(rt), ctypes.byref(rl)))
    ll = ctypes.c_int64()
    ctx.check(ctx.lib.kmb_context_kernel_time(ctx.handle, 3, None, ctypes.byref(ll)))
    gpu_launches = int(ll.value)
    ctx.check(ctx.lib.kmb_context_set_kernel_timing(ctx.handle, 0))
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = iters_done / (ms / 1e3)

    # Plain-form comparison (tensor-core form over plain FP32, target >= 3x) on the same data, when timing the BF16 form.
    plain_value = None
    if tc_form and args.plain_steps > 0:
        C.copy_(C0)
        e0.record(stream)
        p = _native.kmb_params(k, args.plain_steps, 0.0, _native.KMB_FORM_PLAIN, 0)
        it = ctypes.c_int64()
        ctx.check(ctx.lib.kmb_lloyd_iterate(ctx.handle, _native.KMB_F32, X.data_ptr(), n, d, C.data_ptr(),
                                            ctypes.byref(p), labels.data_ptr(), ctypes.byref(it), None))
        e1.record(stream)
        torch.cuda.synchronize()
        plain_value = it.value / (e0.elapsed_time(e1) / 1e3)

    # Roofline of the dominant kernel.
    peaks, peak_src = load_peaks()
    flops_per_launch = 2.0 * n * k * d
    avg_kernel_s = (kt.value / max(kl.value, 1)) / 1e3
    achieved_tflops = flops_per_launch / avg_kernel_s / 1e12 if kl.value else None
    if tc_form:
        peak = peaks["bf16_tflops_sustained"]
        peak_note = f"bf16 dense sustained ({peak_src})"
    else:
        peak = measured_fma_peak_tflops(local, 0)
        peak_note = "FP32 FMA peak measured on this GPU (kmb_measure_fma_peak, larger of scalar and packed-pair FMA)"
    dpad = (d + 63) // 64 * 64
    if tc_form:
        # Xhi (+ Xlo for the split form) read once, labels + d2 written
        algo_bytes = (4 if form == _native.KMB_FORM_BF16X3 else 2) * n * dpad + 8 * n
        # DRAM read+write bytes per row from the ncu capture summarised in
        # profiles/assign_tc_kernel_precision_n1M.txt (scaled by rows).
        traffic = args.traffic_bytes if args.traffic_bytes is not None else TC_DRAM_BYTES_PER_ROW * n
        traffic_src = "ncu dram__bytes_read+write per row of a 1M-row capture, x rows"
    else:
        algo_bytes = 4 * n * d + 8 * n
        traffic = args.traffic_bytes
        traffic_src = None
    roofline = {"bound": "tensor" if tc_form else "fp32_fma", "achieved": achieved_tflops,
                "peak": peak, "unit": "TFLOP/s", "frac": (achieved_tflops / peak) if achieved_tflops else None,
                "traffic": traffic, "traffic_source": traffic_src, "peak_source": peak_note,
                "kernel_ms_avg": avg_kernel_s * 1e3, "kernel_launches": kl.value,
                "update_ms_avg": (ut.value / max(ul.value, 1)),
                "recheck_ms_avg": (rt.value / max(rl.value, 1)) if rl.value else None, "algorithmic_flops_per_launch": flops_per_launch,
                "algorithmic_bytes_per_launch": algo_bytes}

    # e2e through the public API with pinned host buffers.
    e2e = None
    Xh = None
    if rank == 0 and (args.e2e or (world == 1 and args.cpu_iterations > 0)):
        Xh = torch.empty((n, d), dtype=torch.float32, pin_memory=True)
        Xh.copy_(X)
    if rank == 0 and args.e2e:
        C0h = C0.cpu().numpy()
        Xn = Xh.numpy()
        desc = kmeans.descriptor(np.float32).set_cluster_count(k).set_max_iteration_count(args.steps) \
            .set_compute_form(form)
        # one untimed call sizes the context's device workspace (first-call allocations),
        # as the warm-up steps do for the device-resident measurement
        kmeans.train(kmeans.descriptor(np.float32).set_cluster_count(k).set_max_iteration_count(1)
                     .set_compute_form(form), Xn, C0h)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = kmeans.train(desc, Xn, C0h)
        t1 = time.perf_counter()
        T = max(r.get_iteration_count(), 1)
        e2e = {"value": T / (t1 - t0), "unit": UNIT, "h2d_bytes_per_step": (n * d * 4 + k * d * 4) // T,
               "d2h_bytes_per_step": (n * 4 + k * d * 4 + 8) // T,
               "note": "one kmeans.train call on pinned host rows (after one untimed call that sizes the "
                       "workspace): H2D, iterations, final responses + objective, D2H"}

    cpu = None
    if rank == 0 and world == 1 and args.cpu_iterations > 0:
        from oracle import daal_ref
        if daal_ref.available():
            threads = os.cpu_count() or 1
            v, per_iter, it = cpu_reference_iters_per_s(Xh.numpy(), C0.cpu().numpy(), n, args.cpu_iterations,
                                                        threads)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
                   "sample": f"all {n} rows, {it} Lloyd iterations of the reference DAAL kernel (one train call "
                             f"minus its final pass, timed as an infer call; OpenBLAS sgemm, std::thread shim)"}
    del Xh

    plain_scale = None
    if rank == 0 and world == 1 and args.plain_scale:
        plain_scale = run_plain_scale(args, ctx, local)

    plusplus = None
    if rank == 0 and world == 1 and args.plusplus_k > 1:
        plusplus = run_plusplus(args, X, ctx)
    csr = None
    if rank == 0 and world == 1 and args.csr_rows > 0:
        csr = run_csr(args, ctx)

    batched = None
    if rank == 0 and world == 1 and args.batched_problems > 0:
        batched = run_batched(args)
    serving = None
    if rank == 0 and world == 1 and args.serving_requests > 0:
        del X
        torch.cuda.empty_cache()
        serving = run_serving(args, local)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / max(iters_done, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config(n, d, k),
            "form": args.form, "iterations_completed": iters_done,
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": gpu_launches, "clocks": clocks,
            "plain_fp32_value": plain_value,
            "bf16_over_plain": (value / plain_value) if plain_value else None,
            "recheck_rows_per_iteration": st.rechecked_rows / max(iters_done, 1),
            "full_rescans_per_iteration": st.full_rescans / max(iters_done, 1),
            "plain_at_scale": plain_scale,
            "serving": serving,
            "batched": batched,
            "plusplus": plusplus,
            "csr": csr,
        }
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--form", default="bf16x3", choices=["bf16", "bf16x3", "plain"])
    ap.add_argument("--plain-steps", type=int, default=10)
    ap.add_argument("--cpu-iterations", type=int, default=2,
                    help="Lloyd iterations of the reference kernel on all rows for cpu_baseline (0 skips it)")
    ap.add_argument("--cpu-sample-rows", type=int, default=200_000,
                    help="rows of the host-core baselines of the k-means++ and CSR measurements")
    ap.add_argument("--traffic-bytes", type=float, default=None)
    ap.add_argument("--no-e2e", dest="e2e", action="store_false")
    ap.add_argument("--no-plain-scale", dest="plain_scale", action="store_false",
                    help="skip the plain FP32 measurement at n=10M, d=64, k=256")
    ap.add_argument("--batched-problems", type=int, default=4096,
                    help="problems in the batched-form measurement (0 skips it)")
    ap.add_argument("--serving-requests", type=int, default=30000,
                    help="requests per serving load point (0 skips the serving measurement)")
    ap.add_argument("--serving-lanes", type=int, default=4, help="lanes (streams) of the serving engine")
    ap.add_argument("--plain-scale-rows", type=int, default=None,
                    help="rows of the plain-at-scale leg (default: the configured 10,000,000; smaller for profiling)")
    ap.add_argument("--csr-rows", type=int, default=2_000_000,
                    help="rows of the CSR (lloyd_csr) measurement (0 skips it)")
    ap.add_argument("--plusplus-k", type=int, default=1024,
                    help="centers of the k-means++ initialisation measurement (0 skips it)")
    ap.add_argument("--rows", type=int, default=None,
                    help="fewer rows of the same workload (profiling captures); default: the full 20M")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
