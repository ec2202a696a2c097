"""Seeded synthetic workloads for the kNN + smooth-kNN path.

No public dataset is involved: every workload is generated from
``numpy.random.Generator(PCG64(seed))`` in float64 and cast to float32
row-major, in the orders spelled out below.

* ``blobs_1k``      1000 x 50, 10 clusters, centres U[-10,10]^50, sigma 1,
                     100 points per cluster (cluster-major), seed 7; euclidean, k=15.
* ``dups_20k``      20000 x 128, 50 clusters, centres N(0, 4^2 I), per-cluster
                     sigma U[0.5, 2], uniform labels; then 5% of rows become exact
                     copies of other rows and 2% copies with one coordinate moved
                     one ulp toward +inf; euclidean, k=15.
* ``embed_50k``     50000 x 384, N(0, diag(i^-1.2)) plus a shared offset of norm
                     0.3, rows L2-normalised in float64; cosine, k=30.
* ``batch_256``     256 datasets, N log-uniform [200, 8000], d in {16, 50, 128},
                     3-20 clusters, sigma U[0.3, 3], 70/30 euclidean/cosine, k=15,
                     seed 11.
* ``serve_2000``    2000 requests, N log-uniform [500, 50000], d in {32, 64, 300},
                     metric 50/40/10 euclidean/cosine/manhattan, k in {15, 30},
                     Poisson arrivals, one seed per request; the points of a
                     request are a prefix of one of four seeded 50,000-point
                     mixtures of its d (``serve_pool``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


@dataclass
class Workload:
    name: str
    data: np.ndarray  # float32, n x d, C-contiguous
    k: int
    metric: str

    @property
    def n(self) -> int:
        return self.data.shape[0]

    @property
    def d(self) -> int:
        return self.data.shape[1]


def blobs_1k(seed: int = 7) -> Workload:
    g = _rng(seed)
    centres = g.uniform(-10.0, 10.0, size=(10, 50))
    pts = np.concatenate([c + g.normal(0.0, 1.0, size=(100, 50)) for c in centres])
    return Workload("blobs_1k", np.ascontiguousarray(pts.astype(np.float32)), 15, "euclidean")


def gaussian_mixture(g: np.random.Generator, n: int, d: int, clusters: int, centre_scale: float,
                     sigma_lo: float, sigma_hi: float) -> np.ndarray:
    centres = g.normal(0.0, centre_scale, size=(clusters, d))
    sigmas = g.uniform(sigma_lo, sigma_hi, size=clusters)
    labels = g.integers(0, clusters, size=n)
    pts = centres[labels] + g.normal(0.0, 1.0, size=(n, d)) * sigmas[labels, None]
    return pts


def dups_20k(n: int = 20000, d: int = 128, seed: int = 2) -> Workload:
    g = _rng(seed)
    x = gaussian_mixture(g, n, d, 50, 4.0, 0.5, 2.0).astype(np.float32)
    n_dup, n_ulp = int(round(0.05 * n)), int(round(0.02 * n))
    perm = g.permutation(n)
    dup_rows, ulp_rows = perm[:n_dup], perm[n_dup:n_dup + n_ulp]
    sources = perm[n_dup + n_ulp:]  # rows that are never overwritten
    x[dup_rows] = x[g.choice(sources, size=n_dup)]
    src = g.choice(sources, size=n_ulp)
    x[ulp_rows] = x[src]
    coord = g.integers(0, d, size=n_ulp)
    x[ulp_rows, coord] = np.nextafter(x[ulp_rows, coord], np.float32(np.inf))
    return Workload("dups_20k", np.ascontiguousarray(x), 15, "euclidean")


def embedding_like(g: np.random.Generator, n: int, d: int) -> np.ndarray:
    """Rows with an embedding model's shape: N(0, diag(i^-1.2)) plus a shared
    offset of norm 0.3, L2-normalised (float64)."""
    lam = np.arange(1, d + 1, dtype=np.float64) ** -1.2
    z = g.normal(0.0, 1.0, size=(n, d)) * np.sqrt(lam)
    off = g.normal(0.0, 1.0, size=d)
    z += 0.3 * off / np.linalg.norm(off)
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    return z


def embed_50k(n: int = 50000, d: int = 384, seed: int = 3) -> Workload:
    g = _rng(seed)
    lam = np.arange(1, d + 1, dtype=np.float64) ** -1.2
    z = g.normal(0.0, 1.0, size=(n, d)) * np.sqrt(lam)
    off = g.normal(0.0, 1.0, size=d)
    z += 0.3 * off / np.linalg.norm(off)
    z /= np.linalg.norm(z, axis=1, keepdims=True)
    return Workload("embed_50k", np.ascontiguousarray(z.astype(np.float32)), 30, "cosine")


def batch_256(seed: int = 11, count: int = 256) -> list[Workload]:
    g = _rng(seed)
    out = []
    for j in range(count):
        n = int(round(math.exp(g.uniform(math.log(200), math.log(8000)))))
        d = int(g.choice([16, 50, 128]))
        clusters = int(g.integers(3, 21))
        metric = "euclidean" if g.uniform() < 0.7 else "cosine"
        centres = g.uniform(-10.0, 10.0, size=(clusters, d))
        sig = g.uniform(0.3, 3.0, size=clusters)
        labels = g.integers(0, clusters, size=n)
        x = centres[labels] + g.normal(0.0, 1.0, size=(n, d)) * sig[labels, None]
        out.append(Workload(f"batch_{j}", np.ascontiguousarray(x.astype(np.float32)), 15, metric))
    return out


@dataclass
class Request:
    seq: int
    arrival_s: float
    n: int
    d: int
    k: int
    metric: str
    seed: int

    def workload(self) -> Workload:
        g = _rng(self.seed)
        clusters = int(g.integers(3, 21))
        x = gaussian_mixture(g, self.n, self.d, clusters, 4.0, 0.3, 3.0)
        return Workload(f"req_{self.seq}", np.ascontiguousarray(x.astype(np.float32)), self.k,
                        self.metric)

    @property
    def pool_slot(self) -> int:
        return self.seed % SERVE_POOL_SLOTS

    def points(self, pools: dict) -> np.ndarray:
        """The request's n x d points: a prefix of its pool (``serve_pool``);
        ``pools[(d, slot)]`` holds the pool arrays."""
        return pools[(self.d, self.pool_slot)][: self.n]


def serve_2000(rate_per_s: float, count: int = 2000, seed: int = 5000,
               n_lo: int = 500, n_hi: int = 50000) -> list[Request]:
    """Poisson arrivals at ``rate_per_s``; request i is generated from seed + i."""
    g = _rng(seed)
    t = 0.0
    reqs = []
    for i in range(count):
        t += g.exponential(1.0 / rate_per_s)
        n = int(round(math.exp(g.uniform(math.log(n_lo), math.log(n_hi)))))
        d = int(g.choice([32, 64, 300]))
        u = g.uniform()
        metric = "euclidean" if u < 0.5 else ("cosine" if u < 0.9 else "manhattan")
        k = int(g.choice([15, 30]))
        reqs.append(Request(i, t, n, d, k, metric, seed + 1 + i))
    return reqs


SERVE_POOL_SLOTS = 4
SERVE_POOL_N = 50000


def serve_pool(d: int, slot: int, n: int = SERVE_POOL_N) -> np.ndarray:
    """One of the seeded 50,000-point Gaussian mixtures of dimension ``d`` that
    serving requests draw their points from: request i uses the first N rows
    of slot ``(seed + i) % SERVE_POOL_SLOTS`` of its d (a prefix of a mixture
    sample is itself a mixture sample), so 2000 requests need 12 pools, not
    2000 generated datasets."""
    g = _rng(700000 + 10 * d + slot)
    clusters = int(g.integers(3, 21))
    return np.ascontiguousarray(gaussian_mixture(g, n, d, clusters, 4.0, 0.3, 3.0).astype(np.float32))


WORKLOADS = {"blobs_1k": blobs_1k, "dups_20k": dups_20k, "embed_50k": embed_50k}
