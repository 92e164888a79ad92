"""Seeded synthetic k-means workloads (stand-ins for the benchmark data shapes).

No public dataset is used: each generator builds a Gaussian mixture with the
shapes, sizes and value distributions of the corresponding configuration,
deterministically from a seed, with torch generators on the requested device
(CPU for small cases and fixtures, CUDA for the multi-GB benchmark case).

* plain_cpu:  n=100,000, d=20, k=20; 20 isotropic blobs (std 1), centres
  U[-10,10]^20, equal weights; init = first k rows; 50 iterations, eps 0.
* plain_gpu:  n=10,000,000, d=64, k=256; 256 anisotropic blobs (per-blob
  diagonal std log-uniform in [0.3, 3]), centres U[-20,20]^64, weights
  Dirichlet(1); init = seeded uniform row sample; exactly 20 iterations.
* precision:  n=20,000,000, d=128, k=1024; 1024 blobs (std 1), centres
  U[-5,5]^128; 10% of rows on perpendicular bisectors of random centre pairs
  plus N(0, 1e-4) noise (variance 1e-4); init = seeded row sample; 20 iterations.
"""
from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class Workload:
    name: str
    n: int
    d: int
    k: int
    iterations: int
    eps: float
    seed: int


PLAIN_CPU = Workload("plain_cpu", 100_000, 20, 20, 50, 0.0, 1001)
PLAIN_GPU = Workload("plain_gpu", 10_000_000, 64, 256, 20, 0.0, 1002)
PRECISION = Workload("precision", 20_000_000, 128, 1024, 20, 0.0, 1003)


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    return g


def blobs(n, d, k, seed, device="cpu", centre_box=10.0, std=1.0, dtype=torch.float32, chunk=1 << 21):
    """Isotropic Gaussian blobs with equal weights; returns (X, centres)."""
    g = _gen(seed, device)
    centres = (torch.rand(k, d, generator=g, device=device, dtype=torch.float64) * 2 - 1) * centre_box
    X = torch.empty(n, d, dtype=dtype, device=device)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = torch.randint(0, k, (e - s,), generator=g, device=device)
        X[s:e] = (centres[lab] + std * torch.randn(e - s, d, generator=g, device=device, dtype=torch.float64)).to(dtype)
    return X, centres


def anisotropic_blobs(n, d, k, seed, device="cpu", centre_box=20.0, std_range=(0.3, 3.0), dtype=torch.float32,
                      chunk=1 << 21):
    """Blobs with per-blob diagonal std log-uniform in std_range and Dirichlet(1) weights."""
    g = _gen(seed, device)
    centres = (torch.rand(k, d, generator=g, device=device, dtype=torch.float64) * 2 - 1) * centre_box
    lo, hi = torch.log(torch.tensor(std_range[0], dtype=torch.float64)), torch.log(torch.tensor(std_range[1], dtype=torch.float64))
    stds = torch.exp(lo + (hi - lo) * torch.rand(k, d, generator=g, device=device, dtype=torch.float64))
    w = -torch.log(torch.rand(k, generator=g, device=device, dtype=torch.float64))  # Dirichlet(1) = normalised Exp(1)
    w = w / w.sum()
    X = torch.empty(n, d, dtype=dtype, device=device)
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        lab = torch.multinomial(w, e - s, replacement=True, generator=g)
        X[s:e] = (centres[lab] + stds[lab] * torch.randn(e - s, d, generator=g, device=device, dtype=torch.float64)).to(dtype)
    return X, centres


def bisector_blobs(n, d, k, seed, device="cpu", centre_box=5.0, std=1.0, tie_fraction=0.1, noise_var=1e-4,
                   dtype=torch.float32, chunk=1 << 21):
    """Blobs plus `tie_fraction` of rows on perpendicular bisectors of random centre pairs (+ small noise)."""
    g = _gen(seed, device)
    centres = (torch.rand(k, d, generator=g, device=device, dtype=torch.float64) * 2 - 1) * centre_box
    X = torch.empty(n, d, dtype=dtype, device=device)
    noise_std = noise_var ** 0.5
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        m = e - s
        lab = torch.randint(0, k, (m,), generator=g, device=device)
        rows = centres[lab] + std * torch.randn(m, d, generator=g, device=device, dtype=torch.float64)
        tie = torch.rand(m, generator=g, device=device) < tie_fraction
        nt = int(tie.sum())
        if nt:
            a = torch.randint(0, k, (nt,), generator=g, device=device)
            b = (a + torch.randint(1, k, (nt,), generator=g, device=device)) % k
            ca, cb = centres[a], centres[b]
            u = cb - ca
            u = u / u.norm(dim=1, keepdim=True)
            v = std * torch.randn(nt, d, generator=g, device=device, dtype=torch.float64)
            v = v - (v * u).sum(dim=1, keepdim=True) * u
            pts = 0.5 * (ca + cb) + v + noise_std * torch.randn(nt, d, generator=g, device=device, dtype=torch.float64)
            rows[tie] = pts
        X[s:e] = rows.to(dtype)
    return X, centres


def sample_rows(X, k, seed):
    """Seeded uniform sample of k distinct rows (initial centroids)."""
    g = _gen(seed + 7, "cpu")
    idx = torch.randperm(X.shape[0], generator=g)[:k].sort().values
    return X[idx.to(X.device)].clone()


def make(w: Workload, device="cpu", n=None, dtype=torch.float32):
    """(X, C0) for workload w, optionally with fewer rows n (same distribution)."""
    n = w.n if n is None else n
    if w.name == "plain_cpu":
        X, _ = blobs(n, w.d, w.k, w.seed, device, 10.0, 1.0, dtype)
        return X, X[: w.k].clone()
    if w.name == "plain_gpu":
        X, _ = anisotropic_blobs(n, w.d, w.k, w.seed, device, dtype=dtype)
        return X, sample_rows(X, w.k, w.seed)
    if w.name == "precision":
        X, _ = bisector_blobs(n, w.d, w.k, w.seed, device, dtype=dtype)
        return X, sample_rows(X, w.k, w.seed)
    raise KeyError(w.name)
