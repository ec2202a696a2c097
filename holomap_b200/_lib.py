"""ctypes binding of libholomap_cuda.so (the C ABI declared in include/holomap_cuda.h).

This is the Python mirror of the reference's two crate-private calls on the
kNN path (src/api.rs:147-148):

* ``exact_knn(data, n_features, k, metric)`` -> :class:`Knn`   (src/knn.rs:22)
* ``smooth_knn(knn_dists, k)`` -> :class:`SmoothKnn`           (src/smooth_knn.rs:23)

with the same argument meaning, output layout (row-major n x k, self included)
and preconditions (src/api.rs:114-145).  Every call runs on the GPU through the
CUDA library; there is no CPU fallback, and importing a package whose library
has not been built raises at once.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libholomap_cuda.so"

HM_OK = 0
HM_ERR_INVALID = -1
HM_ERR_OOM = -2
HM_ERR_CUDA = -3
HM_ERR_TIMEOUT = -4
HM_ERR_ADMISSION = -5
HM_ERR_UNSUPPORTED = -6
HM_ERR_NOT_READY = -7

ERROR_NAMES = {
    HM_ERR_INVALID: "INVALID", HM_ERR_OOM: "OOM", HM_ERR_CUDA: "CUDA",
    HM_ERR_TIMEOUT: "TIMEOUT", HM_ERR_ADMISSION: "ADMISSION",
    HM_ERR_UNSUPPORTED: "UNSUPPORTED", HM_ERR_NOT_READY: "NOT_READY",
}


class Metric(enum.IntEnum):
    """The reference's ``Metric`` (src/metric.rs:8-15) plus the manhattan
    extension, which has no reference counterpart."""

    EUCLIDEAN = 0
    COSINE = 1
    MANHATTAN = 2

    @classmethod
    def parse(cls, s) -> "Metric":
        """Case-insensitive, like ``FromStr for Metric`` (src/metric.rs:21-30)."""
        if isinstance(s, Metric):
            return s
        if isinstance(s, (int, np.integer)):
            return cls(int(s))
        try:
            return cls[str(s).upper()]
        except KeyError:
            raise ValueError('metric must be "euclidean", "cosine" or "manhattan"') from None

    def __str__(self) -> str:
        return self.name.lower()


class KnnPath(enum.IntEnum):
    """How the N x N distance bulk is evaluated.  Every path returns the same
    bytes; they differ only in speed."""

    AUTO = 0
    PLAIN = 1
    SCREEN_BF16 = 2
    SCREEN_TF32 = 3
    SCREEN_BF16X3 = 4

    @classmethod
    def parse(cls, s) -> "KnnPath":
        if isinstance(s, KnnPath):
            return s
        if isinstance(s, (int, np.integer)):
            return cls(int(s))
        return cls[str(s).upper()]


class HolomapCudaError(RuntimeError):
    """A nonzero status from the C ABI, with hm_last_error()'s message."""

    def __init__(self, code: int, message: str):
        self.code = code
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {message}")


class HolomapInvalidInput(HolomapCudaError, ValueError):
    """HM_ERR_INVALID: the input breaks the reference's preconditions."""


class HmStats(ctypes.Structure):
    _fields_ = [
        ("path_used", ctypes.c_int32),
        ("col_splits", ctypes.c_uint32),
        ("candidates_total", ctypes.c_uint64),
        ("candidates_max_row", ctypes.c_uint32),
        ("candidate_cap", ctypes.c_uint32),
        ("overflow_rows", ctypes.c_uint64),
        ("zero_rho_rows", ctypes.c_uint64),
        ("screen_band", ctypes.c_double),
        ("device_ms", ctypes.c_double),
        ("candidates_emitted", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class HmJob(ctypes.Structure):
    """``hm_job`` of include/holomap_cuda.h (device pointers)."""

    _fields_ = [
        ("data", ctypes.c_void_p),
        ("n", ctypes.c_uint64),
        ("d", ctypes.c_uint32),
        ("k", ctypes.c_uint32),
        ("metric", ctypes.c_int32),
        ("path", ctypes.c_int32),
        ("idx_out", ctypes.c_void_p),
        ("dist_out", ctypes.c_void_p),
        ("sigma_out", ctypes.c_void_p),
        ("rho_out", ctypes.c_void_p),
    ]


class HmCtxConfig(ctypes.Structure):
    """``hm_ctx_config``: device arena bytes, batches in flight, requests per
    batch, the batch's work cap (sum of n*n*d) and the small-request cut
    (n*n*d) below which requests run on high-priority streams; zeros take the
    defaults."""

    _fields_ = [
        ("memory_bytes", ctypes.c_uint64),
        ("max_inflight", ctypes.c_uint32),
        ("max_batch_jobs", ctypes.c_uint32),
        ("max_batch_work", ctypes.c_double),
        ("small_work", ctypes.c_double),
    ]


class HmRequestInfo(ctypes.Structure):
    """``hm_request_info``: status, path, batch and steady-clock times (ms)."""

    _fields_ = [
        ("status", ctypes.c_int32),
        ("path_used", ctypes.c_int32),
        ("batch", ctypes.c_uint64),
        ("batch_jobs", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("submit_ms", ctypes.c_double),
        ("admit_ms", ctypes.c_double),
        ("done_ms", ctypes.c_double),
        ("stats", HmStats),
    ]


class HmCtxTotals(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_uint64),
        ("finished", ctypes.c_uint64),
        ("failed", ctypes.c_uint64),
        ("batches", ctypes.c_uint64),
        ("arena_bytes", ctypes.c_uint64),
        ("arena_peak_bytes", ctypes.c_uint64),
        ("max_batch_jobs_seen", ctypes.c_uint32),
        ("max_inflight_seen", ctypes.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# (name, restype, argtypes) for every symbol of include/holomap_cuda.h
_u64, _u32, _i32, _vp, _sz = (ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                              ctypes.c_size_t)
SIGNATURES = {
    "hm_knn": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _vp, _vp, _vp]),
    "hm_smooth_knn": (_i32, [_vp, _u64, _u32, _vp, _vp]),
    "hm_knn_smooth": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "hm_workspace_bytes": (_sz, [_u64, _u32, _u32, _i32, _i32]),
    "hm_knn_smooth_device": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _vp, _vp, _vp, _vp, _vp,
                                    _sz, _vp, _vp]),
    "hm_stats_from_workspace": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _vp]),
    "hm_smooth_workspace_bytes": (_sz, [_u64]),
    "hm_smooth_knn_device": (_i32, [_vp, _u64, _u32, _vp, _vp, _vp, _vp]),
    "hm_smooth_knn_rows_device": (_i32, [_vp, _u64, _u32, _u64, _u64, _vp, _vp, _vp, _vp]),
    "hm_fuzzy_workspace_bytes": (_sz, [_u64, _u32]),
    "hm_fuzzy_graph_device": (_i32, [_vp, _vp, _vp, _vp, _u64, _u32, _vp, _vp, _vp, _vp, _vp, _sz,
                                     _vp]),
    "hm_fuzzy_graph": (_i32, [_vp, _vp, _vp, _vp, _u64, _u32, _vp, _vp, _vp, _vp]),
    "hm_fuzzy_graph_status": (_i32, [_vp, _u64, _u32, _vp]),
    "hm_laplacian_device": (_i32, [_vp, _vp, _vp, _u64, _u64, _vp, _vp, _vp, _vp]),
    "hm_laplacian_matvec_device": (_i32, [_vp, _vp, _vp, _u64, _vp, _vp, _vp]),
    "hm_eigenpairs_workspace_bytes": (_sz, [_u64, _u32]),
    "hm_eigenpairs_device": (_i32, [_vp, _vp, _vp, _u64, _u32, _vp, _sz, _vp, _vp, _vp, _vp, _vp]),
    "hm_spectral_eigenpairs": (_i32, [_vp, _vp, _vp, _u64, _u64, _u32, _vp, _vp, _vp, _vp]),
    "hm_last_error": (ctypes.c_char_p, []),
    "hm_abi_version": (_i32, []),
    "hm_autotune_path": (_i32, [_u64, _u32, _u32, _i32]),
    "hm_autotune_path_batched": (_i32, [_u64, _u32, _u32, _i32]),
    "hm_tuning_override": (_i32, [_i32]),
    "hm_tuning_symmetric": (_i32, [_i32]),
    "hm_tuning_pair": (_i32, [_i32]),
    "hm_tuning_escalation": (_i32, [_i32]),
    "hm_timing_enable": (_i32, [_i32]),
    "hm_timing_read": (_i32, [_i32, _vp, _vp, _i32]),
    "hm_launch_count": (_u64, []),
    "hm_measure_fp64_rate": (_i32, [_vp]),
    "hm_knn_smooth_noalloc": (_i32, [_vp, _u64, _u32, _u32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "hm_noalloc_scratch_bytes": (_sz, []),
    "hm_noalloc_stats": (_i32, [_vp, _vp]),
    "hm_debug_set_screen_dump": (_i32, [_vp]),
    "hm_debug_tridiag_eigen": (_i32, [_vp, _vp, _u32, _vp, _vp]),
    "hm_batch_create": (_i32, [_vp, _u32, _vp]),
    "hm_batch_destroy": (None, [_vp]),
    "hm_batch_workspace_bytes": (_sz, [_vp]),
    "hm_batch_bind": (_i32, [_vp, _vp, _sz, _vp]),
    "hm_batch_run": (_i32, [_vp, _vp]),
    "hm_batch_graph_launch": (_i32, [_vp, _vp]),
    "hm_batch_job_stats": (_i32, [_vp, _u32, _vp]),
    "hm_batch_job_path": (_i32, [_vp, _u32]),
    "hm_knn_rows_workspace_bytes": (_sz, [_u64, _u32, _u32, _i32, _i32, _u64, _u64]),
    "hm_knn_rows_device": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _u64, _u64, _vp, _vp, _vp, _sz,
                                  _vp, _vp]),
    "hm_knn_rows_stats": (_i32, [_vp, _u64, _u32, _u32, _i32, _i32, _u64, _u64, _vp]),
    "hm_ctx_create": (_i32, [_vp, _vp]),
    "hm_ctx_destroy": (_i32, [_vp]),
    "hm_submit": (_i32, [_vp, _vp, _vp]),
    "hm_poll": (_i32, [_vp, _u64, _vp]),
    "hm_wait": (_i32, [_vp, _u64, _u64, _vp]),
    "hm_release": (_i32, [_vp, _u64]),
    "hm_ctx_totals_read": (_i32, [_vp, _vp]),
}

KCLASS = {"bulk": 0, "select": 1, "smooth": 2, "prep": 3, "exact": 4}


def timing_enable(on: bool = True) -> None:
    check(lib().hm_timing_enable(1 if on else 0))


def timing_read(kclass: str, reset: bool = True) -> tuple[float, int]:
    """(total event-timed ms, launches) of one kernel class since the last reset."""
    ms = ctypes.c_double()
    n = ctypes.c_uint64()
    check(lib().hm_timing_read(KCLASS[kclass], ctypes.byref(ms), ctypes.byref(n), int(reset)))
    return ms.value, n.value


def launch_count() -> int:
    return int(lib().hm_launch_count())


def measure_fp64_rate() -> float:
    """Measured binary64 multiply/add operations per second of the current
    device (a few milliseconds of probe kernels)."""
    r = ctypes.c_double()
    check(lib().hm_measure_fp64_rate(ctypes.byref(r)))
    return r.value

_lib = None


def lib() -> ctypes.CDLL:
    """Load libholomap_cuda.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library first "
                "(python -m holomap_b200.build); there is no CPU fallback")
        L = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != HM_OK:
        msg = lib().hm_last_error().decode(errors="replace")
        if rc == HM_ERR_INVALID:
            raise HolomapInvalidInput(rc, msg)
        raise HolomapCudaError(rc, msg)


@dataclass
class Knn:
    """Mirror of ``Knn`` (src/knn.rs:13-19): row-major n x k."""

    k: int
    indices: np.ndarray  # uint32, n*k
    dists: np.ndarray    # float32, n*k


@dataclass
class SmoothKnn:
    """Mirror of ``SmoothKnn`` (src/smooth_knn.rs:16-19)."""

    sigmas: np.ndarray  # float32, n
    rhos: np.ndarray    # float32, n


def _as_rows(data, n_features: int) -> np.ndarray:
    arr = np.asarray(data)
    if arr.dtype != np.float32:
        raise TypeError("data must be float32 (the reference takes &[f32])")
    flat = np.ascontiguousarray(arr).reshape(-1)
    if n_features <= 0 or flat.size == 0 or flat.size % n_features:
        raise HolomapInvalidInput(
            HM_ERR_INVALID,
            f"data length {flat.size} is not a positive multiple of n_features {n_features}")
    return flat


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def exact_knn(data, n_features: int, k: int, metric="euclidean", path="auto",
              stats: HmStats | None = None) -> Knn:
    """Exact kNN on the GPU; same output as src/knn.rs:22-55."""
    flat = _as_rows(data, n_features)
    n = flat.size // n_features
    idx = np.empty(n * k, dtype=np.uint32)
    dist = np.empty(n * k, dtype=np.float32)
    check(lib().hm_knn(_ptr(flat), n, n_features, k, int(Metric.parse(metric)),
                       int(KnnPath.parse(path)), _ptr(idx), _ptr(dist),
                       ctypes.byref(stats) if stats is not None else None))
    return Knn(k, idx, dist)


def smooth_knn(knn_dists, k: int) -> SmoothKnn:
    """smooth-kNN calibration on the GPU; same output as src/smooth_knn.rs:23-80."""
    d = np.ascontiguousarray(np.asarray(knn_dists, dtype=np.float32)).reshape(-1)
    if k <= 0 or d.size == 0 or d.size % k:
        raise HolomapInvalidInput(HM_ERR_INVALID, "knn_dists is not a non-empty n x k matrix")
    n = d.size // k
    sig = np.empty(n, dtype=np.float32)
    rho = np.empty(n, dtype=np.float32)
    check(lib().hm_smooth_knn(_ptr(d), n, k, _ptr(sig), _ptr(rho)))
    return SmoothKnn(sig, rho)


def knn_smooth(data, n_features: int, k: int, metric="euclidean", path="auto",
               stats: HmStats | None = None, out=None):
    """Both stages of src/api.rs:147-148 with one device round trip.

    ``out`` may supply preallocated (indices, dists, sigmas, rhos) host arrays
    (e.g. pinned memory) that are filled in place."""
    flat = _as_rows(data, n_features)
    n = flat.size // n_features
    if out is None:
        idx = np.empty(n * k, dtype=np.uint32)
        dist = np.empty(n * k, dtype=np.float32)
        sig = np.empty(n, dtype=np.float32)
        rho = np.empty(n, dtype=np.float32)
    else:
        idx, dist, sig, rho = out
    check(lib().hm_knn_smooth(_ptr(flat), n, n_features, k, int(Metric.parse(metric)),
                              int(KnnPath.parse(path)), _ptr(idx), _ptr(dist), _ptr(sig),
                              _ptr(rho), ctypes.byref(stats) if stats is not None else None))
    return Knn(k, idx, dist), SmoothKnn(sig, rho)


@dataclass
class FuzzyGraph:
    """Symmetric membership graph as COO sorted by (row, col) (src/fuzzy.rs:16-22)."""
    n: int
    rows: np.ndarray  # uint32
    cols: np.ndarray  # uint32
    vals: np.ndarray  # float32


def fuzzy_simplicial_set(knn: Knn, calib: SmoothKnn) -> FuzzyGraph:
    """The fuzzy simplicial set on the GPU; same entries and bits as
    src/fuzzy.rs:25-91 (each row's kNN indices must be distinct, as
    exact_knn returns them)."""
    k = knn.k
    idx = np.ascontiguousarray(np.asarray(knn.indices, dtype=np.uint32)).reshape(-1)
    dist = np.ascontiguousarray(np.asarray(knn.dists, dtype=np.float32)).reshape(-1)
    sig = np.ascontiguousarray(np.asarray(calib.sigmas, dtype=np.float32)).reshape(-1)
    rho = np.ascontiguousarray(np.asarray(calib.rhos, dtype=np.float32)).reshape(-1)
    if k <= 0 or idx.size == 0 or idx.size % k or dist.size != idx.size:
        raise HolomapInvalidInput(HM_ERR_INVALID, "knn is not a non-empty n x k graph")
    n = idx.size // k
    if sig.size != n or rho.size != n:
        raise HolomapInvalidInput(HM_ERR_INVALID, "calibration length differs from n")
    if int(idx.max()) >= n:
        raise HolomapInvalidInput(HM_ERR_INVALID, "a kNN index is not below n")
    rows = np.empty(2 * n * k, dtype=np.uint32)
    cols = np.empty(2 * n * k, dtype=np.uint32)
    vals = np.empty(2 * n * k, dtype=np.float32)
    nnz = ctypes.c_uint64(0)
    check(lib().hm_fuzzy_graph(_ptr(idx), _ptr(dist), _ptr(sig), _ptr(rho), n, k, _ptr(rows),
                               _ptr(cols), _ptr(vals), ctypes.byref(nnz)))
    m = nnz.value
    return FuzzyGraph(n, rows[:m].copy(), cols[:m].copy(), vals[:m].copy())


@dataclass
class EigenPairs:
    """k smallest eigenpairs of the normalized Laplacian (src/eigen.rs:20-29):
    values ascending, vectors as a (k, n) array (row j = eigenvector j)."""
    values: np.ndarray   # float64, k
    vectors: np.ndarray  # float64, k x n
    cycles: int


def smallest_eigenpairs(graph: FuzzyGraph, k: int) -> EigenPairs:
    """Lanczos eigenpairs of the graph's normalized Laplacian on the GPU
    (src/sparse.rs:56-71 + src/eigen.rs:95-223)."""
    n = int(graph.n)
    rows = np.ascontiguousarray(graph.rows, dtype=np.uint32)
    cols = np.ascontiguousarray(graph.cols, dtype=np.uint32)
    vals = np.ascontiguousarray(graph.vals, dtype=np.float32)
    if rows.size != cols.size or rows.size != vals.size:
        raise HolomapInvalidInput(HM_ERR_INVALID, "rows, cols and vals differ in length")
    out_v = np.empty(k, dtype=np.float64)
    out_x = np.empty(max(k, 1) * n, dtype=np.float64)
    found = ctypes.c_uint32(0)
    cycles = ctypes.c_uint32(0)
    check(lib().hm_spectral_eigenpairs(_ptr(rows), _ptr(cols), _ptr(vals), n, rows.size, k,
                                       _ptr(out_v), _ptr(out_x), ctypes.byref(found),
                                       ctypes.byref(cycles)))
    f = found.value
    return EigenPairs(out_v[:f].copy(), out_x[: f * n].reshape(f, n).copy(), cycles.value)


def workspace_bytes(n: int, d: int, k: int, metric="euclidean", path="auto") -> int:
    b = lib().hm_workspace_bytes(n, d, k, int(Metric.parse(metric)), int(KnnPath.parse(path)))
    if b == 0:
        check(HM_ERR_INVALID)
    return b


def autotune_path(n: int, d: int, k: int, metric="euclidean", batched: bool = False) -> KnnPath:
    """The path HM_PATH_AUTO takes for a problem alone (or, batched=True, for a
    job planned in a batch of several)."""
    f = lib().hm_autotune_path_batched if batched else lib().hm_autotune_path
    return KnnPath(f(n, d, k, int(Metric.parse(metric))))
