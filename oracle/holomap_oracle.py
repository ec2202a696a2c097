"""ctypes wrapper over the C restatement of holomap's kNN + smooth-kNN path.

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline / reference arm import this module as the checker.  The product
(``holomap_b200``) never imports it.

Functions mirror the reference's crate-private calls:

* :func:`exact_knn`   -- ``exact_knn(data, n_features, k, metric)``  (src/knn.rs:22)
* :func:`smooth_knn`  -- ``smooth_knn(knn_dists, k)``                (src/smooth_knn.rs:23)
* :func:`expf`        -- ``libm::expf`` as used at src/fmath.rs:121
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "holomap_oracle.c"
LIB = HERE / "_build" / "libholomap_oracle.so"

# Flags that keep every binary32/binary64 operation separately rounded, as
# Rust evaluates it: no contraction into FMA, no reassociation.
CFLAGS = ["-O2", "-fPIC", "-shared", "-std=c11", "-Wall", "-ffp-contract=off",
          "-fno-fast-math", "-fexcess-precision=standard", "-pthread"]

METRICS = {"euclidean": 0, "cosine": 1, "manhattan": 2}


def build(force: bool = False) -> Path:
    """Compile the oracle with gcc into oracle/_build/ (skipped when fresh)."""
    LIB.parent.mkdir(parents=True, exist_ok=True)
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    tmp = LIB.with_suffix(f".so.tmp{os.getpid()}")
    subprocess.run(["gcc", *CFLAGS, str(SRC), "-o", str(tmp), "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        sz, fp, u32p = ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p
        L.oracle_exact_knn_rows.argtypes = [fp, sz, sz, sz, ctypes.c_int, sz, sz, u32p, fp]
        L.oracle_exact_knn_rows.restype = ctypes.c_int
        L.oracle_exact_knn_rows_mt.argtypes = [fp, sz, sz, sz, ctypes.c_int, sz, sz, u32p, fp,
                                               ctypes.c_int]
        L.oracle_exact_knn_rows_mt.restype = ctypes.c_int
        L.oracle_smooth_knn.argtypes = [fp, sz, sz, fp, fp]
        L.oracle_smooth_knn.restype = ctypes.c_int
        L.oracle_smooth_knn_rows.argtypes = [fp, sz, sz, ctypes.c_float, fp, fp]
        L.oracle_smooth_knn_rows.restype = ctypes.c_int
        for name in ("oracle_euclidean", "oracle_cosine", "oracle_manhattan"):
            getattr(L, name).argtypes = [fp, fp, sz]
            getattr(L, name).restype = ctypes.c_float
        L.oracle_expf.argtypes = [ctypes.c_float]
        L.oracle_expf.restype = ctypes.c_float
        L.oracle_mean.argtypes = [fp, sz]
        L.oracle_mean.restype = ctypes.c_float
        L.oracle_expf_array.argtypes = [fp, fp, sz]
        L.oracle_expf_array.restype = None
        L.oracle_fuzzy_graph.argtypes = [u32p, fp, fp, fp, sz, sz, u32p, u32p, fp]
        L.oracle_fuzzy_graph.restype = ctypes.c_longlong
        u64p = dp = ctypes.c_void_p
        L.oracle_laplacian.argtypes = [u32p, u32p, fp, sz, sz, u64p, dp, dp]
        L.oracle_laplacian.restype = ctypes.c_int
        L.oracle_laplacian_matvec.argtypes = [u64p, u32p, dp, sz, dp, dp]
        L.oracle_laplacian_matvec.restype = None
        L.oracle_lanczos.argtypes = [u64p, u32p, dp, sz, sz, sz, dp, dp, ctypes.c_void_p]
        L.oracle_lanczos.restype = ctypes.c_longlong
        L.oracle_log2.argtypes = [ctypes.c_double]
        L.oracle_log2.restype = ctypes.c_double
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def metric_code(metric) -> int:
    if isinstance(metric, str):
        return METRICS[metric.lower()]
    return int(metric)


def exact_knn(data: np.ndarray, k: int, metric="euclidean", rows=None, threads: int = 1):
    """Exact kNN of ``data`` (n x d, float32).  ``rows`` = (begin, end) restricts
    the query rows (every row still searches all n points).  Returns
    (indices uint32 [rows x k], dists float32 [rows x k])."""
    data = np.ascontiguousarray(data, dtype=np.float32)
    n, d = data.shape
    r0, r1 = (0, n) if rows is None else rows
    idx = np.empty((r1 - r0, k), dtype=np.uint32)
    dist = np.empty((r1 - r0, k), dtype=np.float32)
    m = metric_code(metric)
    if threads > 1:
        rc = lib().oracle_exact_knn_rows_mt(_ptr(data), n, d, k, m, r0, r1, _ptr(idx),
                                            _ptr(dist), threads)
    else:
        rc = lib().oracle_exact_knn_rows(_ptr(data), n, d, k, m, r0, r1, _ptr(idx), _ptr(dist))
    if rc != 0:
        raise ValueError("oracle_exact_knn rejected its arguments")
    return idx, dist


def smooth_knn(dists: np.ndarray, k: int):
    """(sigmas, rhos), each float32 of length n."""
    dists = np.ascontiguousarray(dists, dtype=np.float32).reshape(-1)
    n = dists.size // k
    sig = np.empty(n, dtype=np.float32)
    rho = np.empty(n, dtype=np.float32)
    if lib().oracle_smooth_knn(_ptr(dists), n, k, _ptr(sig), _ptr(rho)) != 0:
        raise ValueError("oracle_smooth_knn rejected its arguments")
    return sig, rho


def smooth_knn_rows(dists: np.ndarray, k: int, mean_all: float):
    dists = np.ascontiguousarray(dists, dtype=np.float32).reshape(-1)
    n = dists.size // k
    sig = np.empty(n, dtype=np.float32)
    rho = np.empty(n, dtype=np.float32)
    lib().oracle_smooth_knn_rows(_ptr(dists), n, k, float(np.float32(mean_all)), _ptr(sig),
                                 _ptr(rho))
    return sig, rho


def mean(values: np.ndarray) -> np.float32:
    v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    return np.float32(lib().oracle_mean(_ptr(v), v.size))


def distance(a: np.ndarray, b: np.ndarray, metric="euclidean") -> np.float32:
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    name = {0: "oracle_euclidean", 1: "oracle_cosine", 2: "oracle_manhattan"}[metric_code(metric)]
    return np.float32(getattr(lib(), name)(_ptr(a), _ptr(b), a.size))


def expf(x) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.empty_like(x)
    lib().oracle_expf_array(_ptr(x), _ptr(y), x.size)
    return y


def fuzzy_graph(indices: np.ndarray, dists: np.ndarray, sigmas: np.ndarray, rhos: np.ndarray,
                k: int):
    """src/fuzzy.rs:25-91: (rows uint32, cols uint32, vals float32), COO sorted
    by (row, col)."""
    idx = np.ascontiguousarray(indices, dtype=np.uint32).reshape(-1)
    dd = np.ascontiguousarray(dists, dtype=np.float32).reshape(-1)
    sg = np.ascontiguousarray(sigmas, dtype=np.float32).reshape(-1)
    rh = np.ascontiguousarray(rhos, dtype=np.float32).reshape(-1)
    n = idx.size // k
    cap = 2 * n * k
    rows = np.empty(cap, dtype=np.uint32)
    cols = np.empty(cap, dtype=np.uint32)
    vals = np.empty(cap, dtype=np.float32)
    m = lib().oracle_fuzzy_graph(_ptr(idx), _ptr(dd), _ptr(sg), _ptr(rh), n, k, _ptr(rows),
                                 _ptr(cols), _ptr(vals))
    if m < 0:
        raise MemoryError("oracle_fuzzy_graph")
    return rows[:m].copy(), cols[:m].copy(), vals[:m].copy()


def laplacian(rows: np.ndarray, cols: np.ndarray, vals: np.ndarray, n: int):
    """src/sparse.rs:21-35, 56-71: (indptr uint64 n+1, s float64 nnz,
    degrees float64 n) of the (row, col)-sorted COO."""
    r = np.ascontiguousarray(rows, dtype=np.uint32)
    c = np.ascontiguousarray(cols, dtype=np.uint32)
    v = np.ascontiguousarray(vals, dtype=np.float32)
    indptr = np.empty(n + 1, dtype=np.uint64)
    sv = np.empty(max(r.size, 1), dtype=np.float64)
    deg = np.empty(n, dtype=np.float64)
    if lib().oracle_laplacian(_ptr(r), _ptr(c), _ptr(v), n, r.size, _ptr(indptr), _ptr(sv),
                              _ptr(deg)) != 0:
        raise MemoryError("oracle_laplacian")
    return indptr, sv[: r.size], deg


def laplacian_matvec(indptr, cols, svals, x):
    """src/sparse.rs:78-84: y = L x."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    ip = np.ascontiguousarray(indptr, dtype=np.uint64)
    c = np.ascontiguousarray(cols, dtype=np.uint32)
    sv = np.ascontiguousarray(svals, dtype=np.float64)
    lib().oracle_laplacian_matvec(_ptr(ip), _ptr(c), _ptr(sv), x.size, _ptr(x), _ptr(y))
    return y


def lanczos(indptr, cols, svals, n: int, k: int, max_cycles: int = 200):
    """src/eigen.rs:95-238: (values ascending, vectors n x found column-major
    as a (found, n) array, cycles).  max_cycles bounds a timing sample (the
    reference runs up to 200)."""
    ip = np.ascontiguousarray(indptr, dtype=np.uint64)
    c = np.ascontiguousarray(cols, dtype=np.uint32)
    sv = np.ascontiguousarray(svals, dtype=np.float64)
    vals = np.empty(k, dtype=np.float64)
    vecs = np.empty(k * n, dtype=np.float64)
    cyc = ctypes.c_size_t(0)
    f = lib().oracle_lanczos(_ptr(ip), _ptr(c), _ptr(sv), n, k, max_cycles, _ptr(vals), _ptr(vecs),
                             ctypes.byref(cyc))
    if f < 0:
        raise MemoryError("oracle_lanczos")
    return vals[:f], vecs[: f * n].reshape(f, n), cyc.value
